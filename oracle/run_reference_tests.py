"""Pin the CPU oracle by running the reference's own test suite against it.

Test infrastructure only.  The reference's Python package
(python/mojo_poissonrecon) is imported from the read-only reference checkout;
its ctypes loader (`_lib.lib()`, _lib.py:74-90) is pre-seeded with this
directory's `liboracle_mpr.so`, which exports the same `mpr_*` symbols as the
Mojo library.  Then the reference's tests/test_kernels.py and
tests/test_reconstruction.py run unmodified.  The one test that needs
PyMeshLab (tests/test_reconstruction.py:28-62) is deselected: PyMeshLab is
not installed here.

Usage:  python oracle/run_reference_tests.py [/path/to/reference]
Exit status is pytest's.
"""

from __future__ import annotations

import ctypes
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_REFERENCE = "/root/reference"


def install_oracle(lib_path: str) -> None:
    """Make the reference's `lib()` return the oracle library."""
    import mojo_poissonrecon._lib as reference_lib

    cdll = ctypes.CDLL(lib_path)
    for name, (argtypes, restype) in reference_lib._SIGNATURES.items():
        fn = getattr(cdll, name)
        fn.argtypes = argtypes
        fn.restype = restype
    reference_lib._loaded = cdll


class _Plugin:
    def __init__(self, lib_path: str):
        self.lib_path = lib_path

    def pytest_configure(self, config):  # noqa: D401 - pytest hook
        install_oracle(self.lib_path)


def main(argv: list[str]) -> int:
    reference = argv[1] if len(argv) > 1 else DEFAULT_REFERENCE
    lib_path = os.path.join(HERE, "liboracle_mpr.so")
    if not os.path.exists(lib_path):
        raise SystemExit(f"build the oracle first: make -C {HERE}")
    sys.path.insert(0, os.path.join(reference, "python"))
    stub_dir = tempfile.mkdtemp(prefix="pymeshlab_stub_")
    with open(os.path.join(stub_dir, "pymeshlab.py"), "w", encoding="utf8") as stub:
        stub.write("raise_on_use = True\n")
    sys.path.insert(0, stub_dir)
    os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
    sys.dont_write_bytecode = True
    import pytest

    args = [
        "-q",
        "-p",
        "no:cacheprovider",
        "--rootdir",
        stub_dir,
        os.path.join(reference, "tests", "test_kernels.py"),
        os.path.join(reference, "tests", "test_reconstruction.py"),
        "-k",
        "not pymeshlab",
    ]
    return pytest.main(args, plugins=[_Plugin(lib_path)])


if __name__ == "__main__":
    sys.exit(main(sys.argv))
