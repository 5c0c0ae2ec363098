"""Kernel parity through the C ABI: every libpoisson_b200 entry point against
the CPU oracle on the same seeded inputs.  Bit-exact wherever the reference's
arithmetic is order-independent; the two reductions (residual norm,
iso-value) within 1e-13 relative."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _a(x):
    return int(x.ctypes.data)


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mojo_poissonrecon_b200 import _native

    return _native.lib()


_alive = []


def dev(x):
    """Device copy of x, kept referenced for the module's lifetime so that an
    inline dev(x).data_ptr() stays valid while the queued kernel reads it."""
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    _alive.append(t)
    if len(_alive) > 64:
        torch.cuda.synchronize()
        del _alive[:-16]
    return t


def stream():
    return torch.cuda.current_stream().cuda_stream


def ok(status, L):
    assert status == 0, L.pb_last_error().decode()


class WS:
    def __init__(self):
        self.t = None

    def __call__(self, nbytes):
        self.t = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device="cuda")
        return self.t.data_ptr(), self.t.numel()


def edge_points(rng, count):
    pts = rng.random((count, 3))
    pts[:8] = [[0, 0, 0], [1, 1, 1], [1, 0, 0.5], [0.5, 0.5, 0.5], [0, 1, 1], [1, 1, 0], [0.25, 0.75, 1.0],
               [1e-17, 1 - 1e-16, 0.5]]
    return pts


@pytest.mark.parametrize("depth", [0, 1, 5, 8, 19])
def test_octree_codes_bit_exact(L, oracle, depth):
    pts = edge_points(np.random.default_rng(depth), 5000)
    codes = torch.empty((len(pts), depth + 1), dtype=torch.int64, device="cuda")
    ok(L.pb_octree_codes_f64(dev(pts).data_ptr(), len(pts), depth, codes.data_ptr(), stream()), L)
    assert np.array_equal(codes.cpu().numpy(), oracle.octree_codes(pts, depth))


@pytest.mark.parametrize("count,depth", [(1, 3), (7, 0), (200, 7), (5000, 5), (100_000, 8), (3000, 19)])
def test_build_octree_bit_exact(oracle, count, depth):
    from mojo_poissonrecon_b200 import build_octree

    rng = np.random.default_rng(count + depth)
    pts = edge_points(rng, count) if count >= 8 else rng.random((count, 3))
    if count > 100:
        pts[100:150] = pts[0:50]  # duplicate points share leaves
    got = build_octree(pts, depth)
    want = oracle.build_octree(pts, depth)
    for k in ("depth", "morton", "parent", "child_start", "child_count", "point_leaf"):
        assert np.array_equal(getattr(got, k), getattr(want, k)), k


def run_splat(L, pts, nrm, n, conf, spn):
    ws = WS()
    grids = [torch.zeros((n, n, n), dtype=torch.float64, device="cuda") for _ in range(5)]
    acc = torch.zeros(1, dtype=torch.int64, device="cuda")
    ptr, size = ws(L.pb_splat_workspace_size(len(pts), n))
    ok(L.pb_splat_f64(dev(pts).data_ptr(), dev(nrm).data_ptr(), len(pts), n, int(conf),
                      *(g.data_ptr() for g in grids), spn, acc.data_ptr(), ptr, size, stream()), L)
    return [g.cpu().numpy() for g in grids], int(acc.item())


@pytest.mark.parametrize("count,n,conf", [(3, 5, True), (300, 9, True), (2000, 17, False), (20000, 33, True),
                                          (200_000, 65, False)])
def test_splat_bit_exact(L, oracle, count, n, conf):
    rng = np.random.default_rng(count)
    pts = edge_points(rng, count) if count >= 8 else rng.random((count, 3))
    nrm = rng.normal(size=(count, 3))
    if count > 10:
        nrm[5] = 0.0  # a rejected sample
        pts[20:30] = pts[10]  # many samples on one node
    got, acc = run_splat(L, pts, nrm, n, conf, 1.5)
    want = [np.zeros((n, n, n)) for _ in range(5)]
    acc_ref = oracle.lib().mpr_splat_f64(_a(pts), _a(nrm), count, n, int(conf), *(_a(w) for w in want), 1.5)
    assert acc == acc_ref
    for g, w, name in zip(got, want, ("density", "vx", "vy", "vz", "screen")):
        assert np.array_equal(g, w), name


@pytest.mark.parametrize("n", [2, 5, 9, 14, 33, 65])
def test_assemble_relax_residual_bit_exact(L, oracle, n):
    rng = np.random.default_rng(n)
    vx, vy, vz, x, b = (rng.normal(size=(n, n, n)) for _ in range(5))
    screen = rng.random((n, n, n))
    O = oracle.lib()
    rhs_ref = np.empty((n, n, n))
    O.mpr_assemble_f64(_a(vx), _a(vy), _a(vz), _a(screen), _a(rhs_ref), n, 4.0, 0.5)
    rhs = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
    ok(L.pb_assemble_f64(dev(vx).data_ptr(), dev(vy).data_ptr(), dev(vz).data_ptr(), dev(screen).data_ptr(),
                         rhs.data_ptr(), n, 4.0, 0.5, stream()), L)
    assert np.array_equal(rhs.cpu().numpy(), rhs_ref)
    xr = x.copy()
    O.mpr_relax_f64(_a(xr), _a(b), _a(screen), n, 4.0, 3)
    xd = dev(x)
    ok(L.pb_relax_f64(xd.data_ptr(), dev(b).data_ptr(), dev(screen).data_ptr(), n, 4.0, 3, stream()), L)
    assert np.array_equal(xd.cpu().numpy(), xr)
    res_ref = np.empty((n, n, n))
    norm_ref = O.mpr_residual_f64(_a(x), _a(b), _a(screen), _a(res_ref), n, 4.0)
    res = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
    norm = torch.empty(1, dtype=torch.float64, device="cuda")
    ws = WS()
    ptr, size = ws(L.pb_residual_workspace_size(n))
    ok(L.pb_residual_f64(dev(x).data_ptr(), dev(b).data_ptr(), dev(screen).data_ptr(), res.data_ptr(), n, 4.0,
                         norm.data_ptr(), ptr, size, stream()), L)
    assert np.array_equal(res.cpu().numpy(), res_ref)
    assert float(norm.item()) == pytest.approx(norm_ref, rel=1e-13)


@pytest.mark.parametrize("fine_n", [3, 5, 9, 17, 33, 129])
def test_restrict_prolong_bit_exact(L, oracle, fine_n):
    rng = np.random.default_rng(fine_n)
    fine = rng.normal(size=(fine_n,) * 3)
    cn = (fine_n + 1) // 2
    coarse = rng.normal(size=(cn,) * 3)
    O = oracle.lib()
    c_ref = np.empty((cn,) * 3)
    O.mpr_restrict_f64(_a(fine), _a(c_ref), fine_n)
    c = torch.empty((cn,) * 3, dtype=torch.float64, device="cuda")
    ok(L.pb_restrict_f64(dev(fine).data_ptr(), c.data_ptr(), fine_n, stream()), L)
    assert np.array_equal(c.cpu().numpy(), c_ref)
    f_ref = fine.copy()
    O.mpr_prolong_add_f64(_a(coarse), _a(f_ref), fine_n)
    fd = dev(fine)
    ok(L.pb_prolong_add_f64(dev(coarse).data_ptr(), fd.data_ptr(), fine_n, stream()), L)
    assert np.array_equal(fd.cpu().numpy(), f_ref)


@pytest.mark.parametrize("count,n,conf", [(3, 9, 0), (3, 9, 1), (5000, 33, 1), (300_000, 65, 0)])
def test_iso_value(L, oracle, count, n, conf):
    rng = np.random.default_rng(count)
    field = rng.normal(size=(n, n, n))
    pts = edge_points(rng, count) if count >= 8 else rng.random((count, 3))
    nrm = rng.normal(size=(count, 3))
    want = oracle.lib().mpr_iso_value_f64(_a(field), _a(pts), _a(nrm), count, n, conf)
    iso = torch.empty(1, dtype=torch.float64, device="cuda")
    ws = WS()
    ptr, size = ws(L.pb_iso_value_workspace_size(count))
    ok(L.pb_iso_value_f64(dev(field).data_ptr(), dev(pts).data_ptr(), dev(nrm).data_ptr(), count, n, conf,
                          iso.data_ptr(), ptr, size, stream()), L)
    assert float(iso.item()) == pytest.approx(want, rel=1e-13, abs=1e-15)


def sphere_field(n, r=0.3):
    axis = np.linspace(0.0, 1.0, n)
    z, y, x = np.meshgrid(axis, axis, axis, indexing="ij")
    return (x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2 - r * r


@pytest.mark.parametrize("case", ["sphere13", "noisy10", "noisy2", "sphere49", "random65", "sphere130"])
def test_dual_contour_bit_exact(oracle, case, golden_kernels):
    from mojo_poissonrecon_b200 import extract_isosurface

    rng = np.random.default_rng(7)
    field = {
        "sphere13": lambda: sphere_field(13),
        "noisy10": lambda: golden_kernels["dual_noisy10_field"],
        "noisy2": lambda: rng.normal(size=(2, 2, 2)),
        "sphere49": lambda: sphere_field(49),
        "random65": lambda: rng.normal(size=(65, 65, 65)),
        "sphere130": lambda: sphere_field(130, 0.41),
    }[case]()
    iso = 0.1 if case == "noisy10" else 0.0
    density = rng.random(field.shape)
    got = extract_isosurface(field, iso_value=iso, density=density)
    want = oracle.extract(field, iso, density)
    assert np.array_equal(got.vertices, want.vertices)
    assert np.array_equal(got.faces, want.faces)
    assert np.array_equal(got.density, want.density)
    if case == "sphere13":
        assert np.allclose(got.vertices, golden_kernels["dual_sphere13_vertices"], rtol=0, atol=4e-16)
        assert np.array_equal(got.faces, golden_kernels["dual_sphere13_faces"])


def test_dual_partial_capacity_matches_reference_semantics(L, oracle):
    """Capacities below the counts (capi.mojo:961-963, :1057): the first
    `capacity` vertices/faces are written, later active cells keep id 0, and
    the full counts are returned."""
    field = sphere_field(17)
    n = 17
    O = oracle.lib()
    cells = n - 1
    scratch = np.empty((cells + 3) // 4, np.int64)
    d1 = np.zeros(1)
    total = O.mpr_dual_vertices_f64(_a(field), _a(field), n, 0.0, _a(scratch), _a(d1), _a(d1), 0)
    cap = total // 2
    cm_ref = np.empty(cells**3, np.int64)
    v_ref = np.zeros((cap, 3))
    vd_ref = np.zeros(cap)
    assert O.mpr_dual_vertices_f64(_a(field), _a(field), n, 0.0, _a(cm_ref), _a(v_ref), _a(vd_ref), cap) == total
    fd = dev(field)
    cm = torch.empty(cells**3, dtype=torch.int64, device="cuda")
    v = torch.zeros((cap, 3), dtype=torch.float64, device="cuda")
    vd = torch.zeros(cap, dtype=torch.float64, device="cuda")
    cnt = torch.empty(1, dtype=torch.int64, device="cuda")
    ws = WS()
    ptr, size = ws(L.pb_dual_workspace_size(n))
    ok(L.pb_dual_vertices_f64(fd.data_ptr(), fd.data_ptr(), n, 0.0, cm.data_ptr(), v.data_ptr(), vd.data_ptr(), cap,
                              cnt.data_ptr(), ptr, size, stream()), L)
    assert int(cnt.item()) == total
    assert np.array_equal(cm.cpu().numpy(), cm_ref)
    assert np.array_equal(v.cpu().numpy(), v_ref) and np.array_equal(vd.cpu().numpy(), vd_ref)
    # faces with a capacity that cuts the list (odd, to hit the "2 more fit" rule)
    cm_full = np.empty(cells**3, np.int64)
    vf = np.zeros((total, 3))
    vdf = np.zeros(total)
    O.mpr_dual_vertices_f64(_a(field), _a(field), n, 0.0, _a(cm_full), _a(vf), _a(vdf), total)
    dummy = np.zeros(1, np.int64)
    nf = O.mpr_dual_faces_f64(_a(field), n, 0.0, _a(cm_full), _a(dummy), 0)
    fcap = nf // 2 + 1
    f_ref = np.full((fcap, 3), -7, np.int64)
    assert O.mpr_dual_faces_f64(_a(field), n, 0.0, _a(cm_full), _a(f_ref), fcap) == nf
    f = torch.full((fcap, 3), -7, dtype=torch.int64, device="cuda")
    ok(L.pb_dual_faces_f64(fd.data_ptr(), n, 0.0, dev(cm_full).data_ptr(), f.data_ptr(), fcap, cnt.data_ptr(), ptr,
                           size, stream()), L)
    assert int(cnt.item()) == nf
    assert np.array_equal(f.cpu().numpy(), f_ref)


def test_prepare_points_bit_exact(oracle):
    """Row filtering and unit-cube mapping (core.py:73-83, 377-385) on device."""
    from mojo_poissonrecon_b200 import core

    rng = np.random.default_rng(3)
    pts = rng.normal(size=(5000, 3)) * 3 + 1
    nrm = rng.normal(size=(5000, 3))
    pts[3, 1] = np.nan
    nrm[7] = 0.0
    nrm[9, 2] = np.inf
    keep = oracle.valid_rows(pts, nrm)
    unit, origin, width = oracle.normalize(pts[keep], 1.1)
    ctx = core._Context()
    dp, dn, count, fmap = core._prepare(ctx, dev(pts), dev(nrm), 1.1)
    assert count == keep.sum()
    assert np.array_equal(dp.cpu().numpy(), unit)
    assert np.array_equal(dn.cpu().numpy(), nrm[keep])
    m = fmap.cpu().numpy()
    assert np.array_equal(m[:3], origin) and m[3] == width
