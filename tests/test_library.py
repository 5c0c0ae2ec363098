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


def _describe(lib, kind, sides, ptrs, aux=None, clouds=None):
    import numpy as np

    count = len(sides)
    clouds = np.arange(count, dtype=np.int64) if clouds is None else np.asarray(clouds, np.int64)
    sides = np.asarray(sides, np.int64)
    p = np.zeros((count, 12), np.uint64)
    for i, row in enumerate(ptrs):
        p[i, :len(row)] = row
    a = np.zeros((count, 4), np.int64) if aux is None else np.asarray(aux, np.int64)
    nbytes = int(lib.pb_batch_desc_bytes(count))
    raw = np.zeros(nbytes + 64, np.uint8)
    off = (-raw.ctypes.data) % 64
    blocks = ctypes.c_int64(-1)
    status = lib.pb_batch_describe(kind, count, clouds.ctypes.data, sides.ctypes.data, p.ctypes.data, a.ctypes.data,
                                   0, raw[off:].ctypes.data, nbytes, ctypes.byref(blocks))
    return status, blocks.value


def test_batch_descriptors_count_blocks_on_the_host():
    """pb_batch_describe (no GPU needed for the non-TMA kinds): a grouped
    launch's blocks are the sum of each grid's own launch grid."""
    from mojo_poissonrecon_b200 import _native

    lib = _native.lib()
    fake = [0x1000 * (k + 1) for k in range(12)]
    # packed relaxation: grid ((Pc*n + 255)/256, n), Pc = (n+1)/2
    sides = [17, 33, 65, 129]
    status, blocks = _describe(lib, 4, sides, [fake[:7]] * 4)
    assert status == 0, lib.pb_last_error()
    assert blocks == sum(((n + 1) // 2 * n + 255) // 256 * n for n in sides)
    # residual + restriction of level 0: (cn/64, cn/4, cn/4) coarse tiles
    status, blocks = _describe(lib, 3, [257, 33], [fake[:5]] * 2)
    assert status == 0
    assert blocks == sum(-(-c // 64) * -(-c // 4) * -(-c // 4) for c in (129, 17))
    # FCG pass 2: (n/32, n/8, n/24) tiles; pass-1 blocks match pb_batch_fcg_blocks
    status, blocks = _describe(lib, 11, [257], [fake[:10]])
    assert status == 0 and blocks == lib.pb_batch_fcg_blocks(257, 1) == 9 * 33 * 11
    status, blocks = _describe(lib, 9, [65, 257], [fake[:6]] * 2)
    assert blocks == lib.pb_batch_fcg_blocks(65, 0) + lib.pb_batch_fcg_blocks(257, 0)
    # one block per cloud for the reductions and the coarse cycle
    status, blocks = _describe(lib, 10, [65, 257, 33], [fake[:2]] * 3, aux=[[5, 0, 0, 0]] * 3)
    assert status == 0 and blocks == 3
    status, blocks = _describe(lib, 8, [9, 9], [fake[:3]] * 2, aux=[[1, 1, 1, 0]] * 2)
    assert status == 0 and blocks == 2
    assert lib.pb_batch_fcg_partials(257) >= 4 * lib.pb_batch_fcg_blocks(257, 0)


def test_batch_descriptors_reject_bad_grids():
    from mojo_poissonrecon_b200 import _native

    lib = _native.lib()
    fake = [0x1000 * (k + 1) for k in range(12)]
    assert _describe(lib, 4, [17], [fake[:6]])[0] == 1  # a missing operand
    assert _describe(lib, 4, [18], [fake[:7]])[0] == 1  # not 2^k + 1
    assert _describe(lib, 8, [9, 5], [fake[:3]] * 2, aux=[[1, 1, 1, 0]] * 2)[0] == 1  # mixed coarse sides
    assert b"same side" in lib.pb_last_error()
    assert _describe(lib, 8, [9], [fake[:3]], aux=[[65, 1, 1, 0]])[0] == 1  # sweep count out of range
    assert _describe(lib, 99, [9], [fake])[0] == 1
    assert _describe(lib, 4, [17], [fake[:7]], clouds=[-1])[0] == 1
    assert lib.pb_batch_launch(4, None, 1, 1, None, 0, None) == 1


def test_checked_build_exports_the_same_symbols():
    """The bounds-checked variant (libpoisson_b200_checked.so) exports every
    declared symbol and says it is the checked build; the normal library says
    it is not and reports a clear check word without touching a device."""
    from mojo_poissonrecon_b200 import _native, buildlib

    if not os.path.exists(buildlib.CHECKED_LIBRARY):
        pytest.skip("checked library not built (python -m mojo_poissonrecon_b200.buildlib --checked)")
    checked = ctypes.CDLL(buildlib.CHECKED_LIBRARY)
    missing = [s for s in declared_symbols() if not hasattr(checked, s)]
    assert not missing, missing
    assert checked.pb_checked_build() == 1
    lib = _native.lib()
    assert lib.pb_checked_build() == (1 if _native.CHECKED else 0)
    if not _native.CHECKED:
        assert _native.check_word() == 0


def test_check_word_decoding():
    from mojo_poissonrecon_b200 import _native

    site, index = _native.decode_check_word((3 << 56) | 12345)
    assert (site, index) == (3, 12345)
    assert _native.decode_check_word(0) == (0, 0)
