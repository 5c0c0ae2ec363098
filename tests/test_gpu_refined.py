"""The FP32-refined path: its FP32 kernels against the FP64 oracle (FP32
tolerance, written per test), and the defect-corrected solve against the
FP64 solve of the same system.

Tolerances: a FP32 kernel's output is compared with the oracle's FP64 output
on the same (FP32-representable) inputs within rtol 2e-6 of the largest
magnitude; the refined solve must reach ||b - A x|| / ||b|| <= 1e-8 measured in
FP64 and agree with the FP64 solution at equal residual within 1e-6 relative
(max norm)."""

import numpy as np
import pytest

import mg_reference as mg
from padded import from_padded, geometry, ghosts_zero, to_padded

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mojo_poissonrecon_b200 import _native

    return _native.lib()


def _a(x):
    return int(x.ctypes.data)


def setup(L, n, seed):
    rng = np.random.default_rng(seed)
    screen = rng.random((n, n, n)) * (rng.random((n, n, n)) < 0.2)
    rhs = rng.normal(size=(n, n, n)).astype(np.float32).astype(np.float64)
    x = rng.normal(size=(n, n, n)).astype(np.float32).astype(np.float64)
    D = torch.zeros(geometry(L, n)[1], dtype=torch.float32, device="cuda")
    invD, W = torch.zeros_like(D), torch.zeros_like(D)
    s64 = torch.from_numpy(screen).cuda()
    assert L.pb_level_setup_f32(s64.data_ptr(), n, 4.0, D.data_ptr(), invD.data_ptr(), W.data_ptr(),
                                torch.cuda.current_stream().cuda_stream) == 0
    return screen, rhs, x, D, invD, W


@pytest.mark.parametrize("n,z_chunk", [(33, 0), (33, 5), (65, 0), (129, 3), (257, 0), (257, 100), (513, 0)])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_tma_sweep_matches_fp64_relax(L, oracle, n, z_chunk, mode):
    """TMA-staged sweep against the oracle's FP64 relax (mode 2: the scaled
    prolongation is added in place first)."""
    screen, rhs, x, D, invD, W = setup(L, n, 7 * n + mode)
    cn = (n + 1) // 2
    coarse = np.random.default_rng(2).normal(size=(cn,) * 3).astype(np.float32).astype(np.float64)
    start = x.copy() if mode != 1 else np.zeros_like(x)
    if mode == 2:  # the preconditioner's scaled prolongation, weights as set up on the GPU
        start = mg.prolong(start, coarse, from_padded(L, W, n).ravel(), n)
    want = start.copy()
    oracle.lib().mpr_relax_f64(_a(want), _a(rhs), _a(screen), n, 4.0, 1)
    e_in, rhs32, c32 = to_padded(L, x), to_padded(L, rhs.astype(np.float32)), to_padded(L, coarse)
    e_out = torch.zeros_like(e_in)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    if mode == 2:
        assert L.pb_prolong_fac_f32(c32.data_ptr(), e_in.data_ptr(), W.data_ptr(), n, s) == 0
    assert L.pb_sweep_tma_f32(e_in.data_ptr(), e_out.data_ptr(), rhs32.data_ptr(), invD.data_ptr(), n,
                              1 if mode == 1 else 0, z_chunk, status.data_ptr(), s) == 0, \
        L.pb_last_error()
    assert int(status.item()) == 0
    got = from_padded(L, e_out, n)
    assert np.allclose(got, want, rtol=0, atol=2e-6 * np.abs(want).max())
    assert ghosts_zero(L, e_out, n)


@pytest.mark.parametrize("n", [33, 65, 129])
def test_residual_restrict32_matches_restatement(L, oracle, n):
    """Fused level-0 residual + scaled restriction P^T (s r) / 8 against the
    oracle's FP64 residual (capi.mojo:413-470) restricted by the CPU
    restatement; FP32 rounding bounded by the size of the residual's terms,
    which cancel.  Also checks the weights written by the level set-up."""
    screen, rhs, x, D, invD, W = setup(L, n, 3 * n)
    res = np.empty_like(x)
    oracle.lib().mpr_residual_f64(_a(x), _a(rhs), _a(screen), _a(res), n, 4.0)
    s0 = mg.weights(mg.operator7(mg.level0_diagonal(screen, 4.0)), n)
    assert np.abs(from_padded(L, W, n) - s0.reshape(n, n, n)).max() <= 1e-6
    cn = (n + 1) // 2
    want = (mg.trilinear(n).T @ (s0 * res.ravel()) / 8.0).reshape(cn, cn, cn)
    e32, rhs32 = to_padded(L, x), to_padded(L, rhs)
    coarse = torch.zeros(geometry(L, cn)[1], dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert L.pb_residual_restrict_f32(e32.data_ptr(), rhs32.data_ptr(), D.data_ptr(), W.data_ptr(), coarse.data_ptr(),
                                      n, s) == 0
    got = from_padded(L, coarse, cn)
    terms = ((6 + 4 * screen) * (n - 1) ** 2).max() * np.abs(x).max()
    assert np.abs(got - want).max() <= 4e-7 * terms
    assert ghosts_zero(L, coarse, cn)


@pytest.mark.parametrize("precision", ["fp64", "fp32_refined", "fp32_defect"])
def test_tolerance_solves_reach_target(oracle, precision):
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.torus(40_000, seed=3)
    keep = oracle.valid_rows(pts, nrm)
    unit, _, _ = oracle.normalize(pts[keep], 1.1)
    ref = oracle.solve(unit, nrm[keep], depth=6, confidence=True, tol=1e-11, max_cycles=200, octree=False)
    got = mpr.solve_screened_poisson(unit, nrm[keep], depth=6, confidence=True, tol=1e-8, precision=precision)
    # the reported relative residual is measured in FP64 on the returned field
    res = np.empty_like(got.field)
    n = got.field.shape[0]
    r = oracle.lib().mpr_residual_f64(_a(got.field), _a(got.rhs), _a(got.screen), _a(res), n, 4.0)
    assert r / np.linalg.norm(got.rhs) <= 1e-8
    assert got.relative_residual == pytest.approx(r / np.linalg.norm(got.rhs), rel=1e-6)
    err = np.abs(got.field - ref.field).max() / np.abs(ref.field).max()
    assert err <= 1e-6, err
    assert got.iso_value == pytest.approx(ref.iso_value, rel=1e-6)


def test_refined_cycle_counts():
    """The FP32 cycle with Galerkin coarse levels contracts far faster than the
    reference's rediscretised FP64 cycle: defect correction needs under 40% of
    the FP64 V-cycles and FCG(1) no more than defect correction."""
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.torus(100_000, seed=8)
    a = mpr.solve_screened_poisson(*_unit(pts, nrm), depth=7, confidence=True, tol=1e-8, precision="fp64")
    b = mpr.solve_screened_poisson(*_unit(pts, nrm), depth=7, confidence=True, tol=1e-8, precision="fp32_defect")
    c = mpr.solve_screened_poisson(*_unit(pts, nrm), depth=7, confidence=True, tol=1e-8, precision="fp32_refined")
    for sol in (a, b, c):
        assert sol.relative_residual <= 1e-8
    assert b.cycles <= 0.4 * a.cycles, (a.cycles, b.cycles)
    assert c.cycles <= b.cycles, (b.cycles, c.cycles)
    assert c.cycles <= 7, c.cycles
    # Field accuracy is asserted against a tightly converged oracle solve in
    # test_tolerance_solves_reach_target: two solves that each stop at a 1e-8
    # residual can differ by more than that in the field.


def _unit(pts, nrm):
    lo, hi = pts.min(0), pts.max(0)
    w = (hi - lo).max() * 1.1
    return (pts - (0.5 * (lo + hi) - 0.5 * w)) / w, nrm


def test_refined_mesh_matches_fp64_mesh():
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.torus(50_000, seed=4)
    a = mpr.reconstruct(pts, nrm, depth=7, confidence=True, tol=1e-8, precision="fp64")
    b = mpr.reconstruct(pts, nrm, depth=7, confidence=True, tol=1e-8, precision="fp32_refined")
    assert abs(a.faces.shape[0] - b.faces.shape[0]) <= 0.001 * a.faces.shape[0]
    assert b.iso_value == pytest.approx(a.iso_value, rel=1e-6)


def test_engine_graphs_replay_new_inputs():
    """An engine captures its prologue and iteration graphs on the first solve
    and replays them afterwards: a second system solved on the same engine
    gives the same field, bit for bit, as that system on a fresh engine."""
    from mojo_poissonrecon_b200 import _native as nat
    from mojo_poissonrecon_b200 import solver32

    n = 65
    rng = np.random.default_rng(11)
    systems = []
    for _ in range(2):
        screen = torch.from_numpy(rng.random((n, n, n)) * (rng.random((n, n, n)) < 0.1)).cuda()
        rhs = torch.from_numpy(rng.normal(size=(n, n, n))).cuda()
        systems.append((rhs, screen))
    ws = nat.Workspace(torch.device("cuda"))
    solver32.clear_engines()
    solver32.solve_refined(*systems[0], 4.0, ws)  # captures the graphs
    replayed, stats = solver32.solve_refined(*systems[1], 4.0, ws)
    assert stats.relative_residual <= 1e-8
    solver32.clear_engines()
    fresh, _ = solver32.solve_refined(*systems[1], 4.0, ws)
    assert torch.equal(replayed, fresh)


@pytest.mark.parametrize("n", [33, 65, 257])
def test_sweep_variants_bit_identical(L, n):
    """The sweep's autotuned variants (shared-ring depth, resident blocks per SM,
    rows grouped by parity per warp, one barrier per plane) and z chunks (odd and
    even chunk starts) compute the same bits as the built-in launch shape."""
    from mojo_poissonrecon_b200 import tune

    screen, rhs, x, D, invD, W = setup(L, n, 31 * n)
    e_in = to_padded(L, x.astype(np.float32))
    r32 = to_padded(L, rhs.astype(np.float32))
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream

    def sweep(mode):
        out = torch.zeros_like(e_in)
        assert L.pb_sweep_tma_f32(e_in.data_ptr(), out.data_ptr(), r32.data_ptr(), invD.data_ptr(), n, mode, 0,
                                  status.data_ptr(), s) == 0
        return out

    L.pb_tune_clear()
    try:
        want = [sweep(0), sweep(1)]
        for variant in range(1, 9):
            for z_chunk in (0, 4, 5, 17):
                L.pb_tune_set(tune.SWEEP_VARIANT, n, variant)
                L.pb_tune_set(tune.SWEEP_Z_CHUNK, n, z_chunk)
                got = [sweep(0), sweep(1)]
                assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1]), (variant, z_chunk)
        assert int(status.item()) == 0
    finally:
        L.pb_tune_clear()


@pytest.mark.parametrize("n", [65, 257])
def test_residual_restrict_variants_bit_identical(L, n):
    """The paired variant and other coarse planes per block compute the same bits."""
    from mojo_poissonrecon_b200 import tune

    screen, rhs, x, D, invD, W = setup(L, n, 17 * n)
    e = to_padded(L, x.astype(np.float32))
    r32 = to_padded(L, rhs.astype(np.float32))
    cn = (n + 1) // 2
    s = torch.cuda.current_stream().cuda_stream

    def run():
        out = torch.zeros(geometry(L, cn)[1], dtype=torch.float32, device="cuda")
        assert L.pb_residual_restrict_f32(e.data_ptr(), r32.data_ptr(), D.data_ptr(), W.data_ptr(), out.data_ptr(),
                                          n, s) == 0
        return out

    L.pb_tune_clear()
    try:
        want = run()
        for variant in (0, 1, 3):
            for planes in (0, 1, 3, 8):
                L.pb_tune_set(tune.RESTRICT_VARIANT, n, variant)
                L.pb_tune_set(tune.RESTRICT_PLANES, n, planes)
                assert torch.equal(run(), want), (variant, planes)
    finally:
        L.pb_tune_clear()


@pytest.mark.parametrize("n", [33, 65, 129, 257])
def test_residual_restrict_tma_bit_identical(L, n):
    """The TMA-staged residual-restriction computes the plain kernel's bits at
    every coarse-planes-per-block value, and no bounded wait gives up."""
    from mojo_poissonrecon_b200 import tune

    screen, rhs, x, D, invD, W = setup(L, n, 23 * n)
    e = to_padded(L, x.astype(np.float32))
    r32 = to_padded(L, rhs.astype(np.float32))
    cn = (n + 1) // 2
    s = torch.cuda.current_stream().cuda_stream
    status = torch.zeros(1, dtype=torch.int32, device="cuda")

    def out():
        return torch.full((geometry(L, cn)[1],), float("nan"), dtype=torch.float32, device="cuda")

    L.pb_tune_clear()
    try:
        want = torch.zeros(geometry(L, cn)[1], dtype=torch.float32, device="cuda")
        assert L.pb_residual_restrict_f32(e.data_ptr(), r32.data_ptr(), D.data_ptr(), W.data_ptr(), want.data_ptr(),
                                          n, s) == 0
        want = from_padded(L, want, cn)
        for planes in (0, 1, 3, 8, cn):
            L.pb_tune_set(tune.RESTRICT_PLANES, n, planes)
            got = out()
            assert L.pb_residual_restrict_tma_f32(e.data_ptr(), r32.data_ptr(), D.data_ptr(), W.data_ptr(),
                                                  got.data_ptr(), n, status.data_ptr(), s) == 0
            assert np.array_equal(from_padded(L, got, cn), want), planes
        assert int(status.item()) == 0
    finally:
        L.pb_tune_clear()


def test_residual_restrict_tma_rejects_bad_sides(L):
    t = torch.zeros(64, dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for n in (17, 31, 34, 4099):
        assert L.pb_residual_restrict_tma_f32(t.data_ptr(), t.data_ptr(), t.data_ptr(), t.data_ptr(), t.data_ptr(),
                                              n, status.data_ptr(), s) != 0
