"""The C-ABI library builds, loads without a GPU, and exports every symbol that
include/poisson_b200.h declares; host-side argument checks fail before any
device work."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "poisson_b200.h")


def declared_symbols():
    text = open(HEADER, encoding="utf8").read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pb_\w+)\s*\(", text)))


def test_header_declares_the_reference_operations():
    names = declared_symbols()
    # One GPU entry point per reference symbol (_lib.py:20-32).
    for op in ("pb_init", "pb_octree_codes_f64", "pb_splat_f64", "pb_assemble_f64", "pb_relax_f64",
               "pb_residual_f64", "pb_restrict_f64", "pb_prolong_add_f64", "pb_iso_value_f64",
               "pb_dual_vertices_f64", "pb_dual_faces_f64"):
        assert op in names


def test_library_exports_every_declared_symbol():
    from mojo_poissonrecon_b200 import _native

    lib = _native.lib()
    cdll = ctypes.CDLL(_native.library_path())
    missing = [s for s in declared_symbols() if not hasattr(cdll, s)]
    assert not missing, missing
    # ... and the Python binding table covers the same set.
    assert set(declared_symbols()) <= set(_native.exported_symbols())
    assert lib.pb_version() == 10000


def test_workspace_queries_are_host_only():
    from mojo_poissonrecon_b200 import _native

    lib = _native.lib()
    assert lib.pb_splat_workspace_size(1000, 33) > 8 * 1000 * 16
    assert lib.pb_octree_workspace_size(1000, 8) > 1000 * 16
    assert lib.pb_dual_workspace_size(257) > 0
    assert lib.pb_residual_workspace_size(257) > 0
    assert lib.pb_iso_value_workspace_size(10) > 0
    assert lib.pb_prepare_workspace_size(10) > 0


@pytest.mark.parametrize(
    "call,needle",
    [
        (lambda L: L.pb_relax_f64(None, None, None, 1, 4.0, 1, None), "n must be >= 2"),
        (lambda L: L.pb_restrict_f64(None, None, 1, None), "n must be >= 2"),
        (lambda L: L.pb_octree_codes_f64(None, 5, 20, None, None), "depth"),
        (lambda L: L.pb_splat_f64(None, None, 10, 1, 0, None, None, None, None, None, 1.5, None, None, 0, None),
         "n must be >= 2"),
        (lambda L: L.pb_splat_f64(1, 1, 10, 9, 0, 1, 1, 1, 1, 1, 1.5, 1, None, 0, None), "workspace"),
        (lambda L: L.pb_dual_vertices_f64(None, None, 1, 0.0, None, None, None, 0, None, None, 0, None), "n must"),
    ],
)
def test_invalid_arguments_rejected_before_launch(call, needle):
    from mojo_poissonrecon_b200 import _native

    L = _native.lib()
    status = call(L)
    assert status != 0
    assert needle in L.pb_last_error().decode()


def test_build_entry_compiles_sm100a():
    from mojo_poissonrecon_b200 import buildlib

    assert buildlib.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.exists(buildlib.build())
