"""The allocation-free active-cell count (pb_dual_vertex_count_f64_noalloc).

It serves callers that cannot allocate device memory — for example a serving
loop that must not hit cudaMalloc/cudaFree (they can block or synchronise the
device) or a foreign-language binding that only receives buffers from another
framework's pool.  Its answer must equal the workspace-based count mode of
pb_dual_vertices_f64 exactly (an integer count), on consecutive calls that
reuse its fixed scratch array.  This file is collected last on purpose."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mojo_poissonrecon_b200 import _native

    return _native.lib()


def sphere_field(n, r):
    axis = np.linspace(0.0, 1.0, n)
    z, y, x = np.meshgrid(axis, axis, axis, indexing="ij")
    return np.ascontiguousarray((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2 - r * r)


def workspace_count(L, field_d, n, iso):
    ws = torch.empty(int(L.pb_dual_workspace_size(n)), dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    status = L.pb_dual_vertices_f64(field_d.data_ptr(), field_d.data_ptr(), n, iso, None, None, None, 0,
                                    count.data_ptr(), ws.data_ptr(), ws.numel(), s)
    assert status == 0, L.pb_last_error().decode()
    return int(count.item())


def noalloc_count(L, field_d, n, iso):
    count = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    status = L.pb_dual_vertex_count_f64_noalloc(field_d.data_ptr(), n, iso, count.data_ptr(),
                                                torch.cuda.current_stream().cuda_stream)
    assert status == 0, L.pb_last_error().decode()
    return int(count.item())


def test_noalloc_count_equals_workspace_count_on_consecutive_calls(L):
    rng = np.random.default_rng(5)
    cases = [
        (torch.from_numpy(sphere_field(257, 0.37)).cuda(), 257, 0.0),   # large, many tiles
        (torch.from_numpy(rng.normal(size=(33, 33, 33))).cuda(), 33, 0.1),  # small, after a large one
        (torch.from_numpy(sphere_field(513, 0.41)).cuda(), 513, 0.0),   # the largest accepted side
        (torch.from_numpy(rng.normal(size=(2, 2, 2))).cuda(), 2, 0.0),
    ]
    for field_d, n, iso in cases:
        want = workspace_count(L, field_d, n, iso)
        first = noalloc_count(L, field_d, n, iso)
        second = noalloc_count(L, field_d, n, iso)
        assert first == want and second == want, (n, want, first, second)


def test_noalloc_count_rejects_grids_beyond_its_scratch(L):
    field = torch.zeros(8, dtype=torch.float64, device="cuda")  # never read: rejected before launch
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    # 514 is the first side past the limit (65,918 tiles of 2048 cells against 65,536
    # slots); 1025 and 1 << 40 are far past it (the latter would overflow n^3).
    for n in (514, 1025, 1 << 40):
        status = L.pb_dual_vertex_count_f64_noalloc(field.data_ptr(), n, 0.0, count.data_ptr(),
                                                    torch.cuda.current_stream().cuda_stream)
        assert status == 1, n
        assert "n <= 513" in L.pb_last_error().decode(), n
