"""Bit-array extraction used by reconstruct() (pb_extract_count_f64 /
pb_extract_emit_f64) against the reference-shaped dual-contouring entry points
(pb_dual_vertices_f64 / pb_dual_faces_f64, pinned to the oracle elsewhere):
identical vertex, density and face arrays, bit for bit."""

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


def stream():
    return torch.cuda.current_stream().cuda_stream


def reference_shaped(L, field, density, iso):
    n = field.shape[0]
    ws = torch.empty(L.pb_dual_workspace_size(n), dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    isot = torch.tensor([iso], dtype=torch.float64, device="cuda")
    assert L.pb_dual_vertices_f64_isoptr(field.data_ptr(), density.data_ptr(), n, isot.data_ptr(), None, None, None,
                                         0, count.data_ptr(), ws.data_ptr(), ws.numel(), stream()) == 0
    nv = int(count.item())
    cm = torch.empty(max((n - 1) ** 3, 1), dtype=torch.int64, device="cuda")
    v = torch.empty((nv, 3), dtype=torch.float64, device="cuda")
    vd = torch.empty(nv, dtype=torch.float64, device="cuda")
    if nv:
        assert L.pb_dual_vertices_f64_isoptr(field.data_ptr(), density.data_ptr(), n, isot.data_ptr(),
                                             cm.data_ptr(), v.data_ptr(), vd.data_ptr(), nv, count.data_ptr(),
                                             ws.data_ptr(), ws.numel(), stream()) == 0
    else:
        cm.fill_(-1)
    fc = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert L.pb_dual_faces_f64_isoptr(field.data_ptr(), n, isot.data_ptr(), cm.data_ptr(), None, 0, fc.data_ptr(),
                                      ws.data_ptr(), ws.numel(), stream()) == 0
    nf = int(fc.item())
    f = torch.empty((nf, 3), dtype=torch.int64, device="cuda")
    if nf:
        assert L.pb_dual_faces_f64_isoptr(field.data_ptr(), n, isot.data_ptr(), cm.data_ptr(), f.data_ptr(), nf,
                                          fc.data_ptr(), ws.data_ptr(), ws.numel(), stream()) == 0
    return v.cpu().numpy(), vd.cpu().numpy(), f.cpu().numpy()


def bit_array(L, field, density, iso):
    n = field.shape[0]
    ws = torch.empty(L.pb_extract_workspace_size(n), dtype=torch.uint8, device="cuda")
    counts = torch.empty(2, dtype=torch.int64, device="cuda")
    isot = torch.tensor([iso], dtype=torch.float64, device="cuda")
    assert L.pb_extract_count_f64(field.data_ptr(), n, isot.data_ptr(), counts.data_ptr(), ws.data_ptr(), ws.numel(),
                                  stream()) == 0, L.pb_last_error()
    nv, nf = (int(c) for c in counts.cpu())
    v = torch.empty((nv, 3), dtype=torch.float64, device="cuda")
    vd = torch.empty(nv, dtype=torch.float64, device="cuda")
    f = torch.empty((nf, 3), dtype=torch.int64, device="cuda")
    if nv:
        assert L.pb_extract_emit_f64(field.data_ptr(), density.data_ptr(), n, isot.data_ptr(), v.data_ptr(),
                                     vd.data_ptr(), f.data_ptr() if nf else None, ws.data_ptr(), ws.numel(),
                                     stream()) == 0
    return v.cpu().numpy(), vd.cpu().numpy(), f.cpu().numpy()


def fields():
    rng = np.random.default_rng(5)
    for n in (2, 3, 5, 17, 33, 66, 129):
        yield f"normal{n}", rng.normal(size=(n,) * 3), 0.0
    z, y, x = np.meshgrid(*(np.linspace(-1, 1, 97),) * 3, indexing="ij")
    yield "sphere97", np.sqrt(x * x + y * y + z * z) - 0.6, 0.0
    yield "ties", np.round(rng.normal(size=(33,) * 3), 1), 0.1  # values equal to the iso-value
    yield "constant", np.full((17,) * 3, 2.0), 0.5  # no vertices
    z, y, x = np.meshgrid(*(np.linspace(-1, 1, 257),) * 3, indexing="ij")
    yield "torus257", np.sqrt((np.sqrt(x * x + y * y) - 0.5) ** 2 + z * z) - 0.2, 0.0


@pytest.mark.parametrize("name,field,iso", list(fields()), ids=lambda v: v if isinstance(v, str) else "")
def test_bit_array_extraction_is_identical(L, name, field, iso):
    f = torch.from_numpy(np.ascontiguousarray(field)).cuda()
    dens = torch.from_numpy(np.random.default_rng(1).random(field.shape)).cuda()
    a = reference_shaped(L, f, dens, iso)
    b = bit_array(L, f, dens, iso)
    for u, w in zip(a, b):
        assert u.shape == w.shape
        assert np.array_equal(u.view(np.uint8), w.view(np.uint8)) if u.size else True


def test_two_runs_reuse_workspace(L):
    """count/emit twice on the same workspace with different fields."""
    rng = np.random.default_rng(9)
    for seed in range(2):
        field = torch.from_numpy(rng.normal(size=(33,) * 3)).cuda()
        dens = torch.from_numpy(rng.random((33,) * 3)).cuda()
        a, b = reference_shaped(L, field, dens, 0.0), bit_array(L, field, dens, 0.0)
        for u, w in zip(a, b):
            assert np.array_equal(u, w)
