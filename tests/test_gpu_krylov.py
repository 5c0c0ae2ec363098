"""The FP64 kernels of the refined solvers, each alone against a NumPy restatement.

pb_defect_f64 (r = b - A x, optionally after x_new = x_old + e), and the two
FCG(1) passes: pb_fcg_direction_f64 (the four inner products (z, Az),
(Az, p_prev), (z, r), (p_prev, r) and the step's beta, (p, Ap), alpha, (p, r))
and pb_fcg_update_f64 (p_new = z - beta p_prev, x_new = x + alpha p_new,
r = b - A x_new, ||r||^2), on small odd sides, first and later steps, both
buffer parities.  A is the reference's operator (capi.mojo:282-306, 413-553):
(A x)_i = (deg_i + pw s_i) h^2 x_i - h^2 sum of in-grid neighbours, h = n - 1.

Tolerances: x_new within 4 eps of the magnitudes it is formed from
(|x| + |alpha| (|z| + |beta p|): the update may fuse multiply-adds), p_new within
one FP32 ulp; residuals within 1e-12 of the largest
term of A x (the neighbour sum cancels); inner products and their quotients
within 1e-11 relative (a parallel tree sum against NumPy's pairwise sum)."""

import numpy as np
import pytest

from padded import from_padded, geometry, to_padded

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SIDES = (9, 33, 65)


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mojo_poissonrecon_b200 import _native

    return _native.lib()


def stream():
    return torch.cuda.current_stream().cuda_stream


def apply_A(x, screen, pw):
    """The reference's screened Laplacian with Neumann degrees (capi.mojo:282-306)."""
    n = x.shape[0]
    h2 = float(n - 1) ** 2
    s = np.zeros_like(x)
    deg = np.zeros_like(x)
    for axis in range(3):
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axis] = slice(0, n - 1)
        hi[axis] = slice(1, n)
        s[tuple(lo)] += x[tuple(hi)]
        s[tuple(hi)] += x[tuple(lo)]
        deg[tuple(lo)] += 1
        deg[tuple(hi)] += 1
    return (deg * h2 + pw * screen * h2) * x - s * h2, (deg * h2 + pw * screen * h2) * np.abs(x) + np.abs(s) * h2


def system(n, seed):
    rng = np.random.default_rng(seed)
    screen = rng.random((n, n, n)) * (rng.random((n, n, n)) < 0.3)
    b = rng.normal(size=(n, n, n))
    x = rng.normal(size=(n, n, n))
    return screen, b, x


def f32(a):
    return a.astype(np.float32).astype(np.float64)


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype).cuda()


def check_residual(got, want, scale, what):
    err = np.abs(got - want).max()
    assert err <= 1e-12 * scale.max(), (what, err, scale.max())


@pytest.mark.parametrize("n", SIDES)
@pytest.mark.parametrize("update", [False, True])
def test_defect_matches_restatement(L, n, update):
    pw = 4.0
    screen, b, x = system(n, 100 + n)
    e = f32(np.random.default_rng(n).normal(size=(n, n, n)) * 1e-3)
    x_new_want = x + e if update else x
    r_want, scale = apply_A(x_new_want, screen, pw)
    r_want = b - r_want
    ws = torch.empty(int(L.pb_defect_workspace_size(n)), dtype=torch.uint8, device="cuda")
    r32 = torch.zeros(geometry(L, n)[1], dtype=torch.float32, device="cuda")
    r64 = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
    norm2 = torch.empty(1, dtype=torch.float64, device="cuda")
    dx, db, ds = dev(x), dev(b), dev(screen)
    de = to_padded(L, e.astype(np.float32)) if update else None
    dxn = torch.empty_like(dx) if update else None
    status = L.pb_defect_f64(dx.data_ptr(), de.data_ptr() if update else None, dxn.data_ptr() if update else None,
                             db.data_ptr(), ds.data_ptr(), n, pw, r32.data_ptr(), r64.data_ptr(), norm2.data_ptr(),
                             ws.data_ptr(), ws.numel(), stream())
    assert status == 0, L.pb_last_error().decode()
    if update:
        assert np.array_equal(dxn.cpu().numpy(), x_new_want)  # one FP64 add per node, exact
    check_residual(r64.cpu().numpy(), r_want, scale, "r64")
    assert np.array_equal(from_padded(L, r32, n), f32(r64.cpu().numpy()))
    assert float(norm2.item()) == pytest.approx(float(np.sum(r64.cpu().numpy() ** 2)), rel=1e-11)
    assert float(norm2.item()) == pytest.approx(float(np.sum(r_want ** 2)), rel=1e-9)


def fcg_state(L, n, seed):
    """A mid-solve FCG state: z and r32 padded FP32, p0/p1 dense FP32, x0/x1 FP64."""
    rng = np.random.default_rng(seed)
    screen, b, x = system(n, seed)
    z = f32(rng.normal(size=(n, n, n)))
    r = f32(rng.normal(size=(n, n, n)))
    p = [f32(rng.normal(size=(n, n, n))) for _ in range(2)]
    return screen, b, x, z, r, p


def direction_restated(z, r, p_prev, screen, pw, first, pap_prev):
    az, _ = apply_A(z, screen, pw)
    zz, zr = float(np.sum(z * az)), float(np.sum(z * r))
    zq = 0.0 if first else float(np.sum(az * p_prev))
    pr = 0.0 if first else float(np.sum(p_prev * r))
    beta = 0.0 if first or not pap_prev > 0 else zq / pap_prev
    pap = zz if first else zz - 2.0 * beta * zq + beta * beta * pap_prev
    prn = zr if first else zr - beta * pr
    return pap, beta, (prn / pap if pap > 0 else 0.0), prn


@pytest.mark.parametrize("n", SIDES)
@pytest.mark.parametrize("first,it", [(True, 0), (False, 1), (False, 2)])
def test_fcg_direction_matches_restatement(L, n, first, it):
    pw = 4.0
    screen, _, _, z, r, p = fcg_state(L, n, 7 * n + it)
    # (p_prev, A p_prev) from the previous step: a positive value of the right size
    pap_prev = float(np.sum(p[it & 1] * apply_A(p[it & 1], screen, pw)[0]))
    scal = torch.zeros(8, dtype=torch.float64, device="cuda")
    scal[0] = pap_prev
    flags = torch.tensor([int(first), it, 0, 0], dtype=torch.int32, device="cuda")
    ws = torch.empty(int(L.pb_fcg_workspace_size(n)), dtype=torch.uint8, device="cuda")
    dz, dr = to_padded(L, z.astype(np.float32)), to_padded(L, r.astype(np.float32))
    dp = [dev(a, torch.float32) for a in p]
    ds = dev(screen)
    status = L.pb_fcg_direction_f64(dz.data_ptr(), dp[0].data_ptr(), dp[1].data_ptr(), dr.data_ptr(), ds.data_ptr(),
                                    n, pw, scal.data_ptr(), flags.data_ptr(), ws.data_ptr(), ws.numel(), stream())
    assert status == 0, L.pb_last_error().decode()
    got = scal.cpu().numpy()
    want = direction_restated(z, r, p[it & 1], screen, pw, first, pap_prev)
    names = ("(p, Ap)", "beta", "alpha", "(p, r)")
    for k in range(4):
        assert got[k] == pytest.approx(want[k], rel=1e-11, abs=1e-300), names[k]
    if first:
        assert got[1] == 0.0


@pytest.mark.parametrize("n", SIDES)
@pytest.mark.parametrize("first,it", [(True, 0), (False, 1), (False, 2)])
def test_fcg_update_matches_restatement(L, n, first, it):
    pw = 4.0
    screen, b, x, z, _, p = fcg_state(L, n, 11 * n + it)
    beta, alpha = (0.0 if first else 0.37), 0.81
    odd = it & 1
    scal = torch.tensor([1.0, beta, alpha, 0.0, -1.0, 0, 0, 0], dtype=torch.float64, device="cuda")
    flags = torch.tensor([int(first), it, 0, 0], dtype=torch.int32, device="cuda")
    ws = torch.empty(int(L.pb_fcg_workspace_size(n)), dtype=torch.uint8, device="cuda")
    dz = to_padded(L, z.astype(np.float32))
    dp = [dev(a, torch.float32) for a in p]
    xs = [dev(x), torch.full((n, n, n), np.nan, dtype=torch.float64, device="cuda")]
    if odd:
        xs.reverse()  # the current iterate lives in x[it & 1]
    db, ds = dev(b), dev(screen)
    r32 = torch.zeros(geometry(L, n)[1], dtype=torch.float32, device="cuda")
    status = L.pb_fcg_update_f64(dz.data_ptr(), dp[0].data_ptr(), dp[1].data_ptr(), xs[0].data_ptr(),
                                 xs[1].data_ptr(), db.data_ptr(), ds.data_ptr(), r32.data_ptr(), n, pw,
                                 scal.data_ptr(), flags.data_ptr(), ws.data_ptr(), ws.numel(), stream())
    assert status == 0, L.pb_last_error().decode()
    direction = z - beta * p[odd] if not first else z.copy()
    x_want = x + alpha * direction
    x_got = xs[1 - odd].cpu().numpy()
    # the kernel may fuse z - beta p and x + alpha d into multiply-adds: each rounding is
    # relative to the magnitudes before cancellation, |x| + |alpha| (|z| + |beta p|)
    scale = np.abs(x) + abs(alpha) * (np.abs(z) + abs(beta) * np.abs(p[odd]))
    assert np.all(np.abs(x_got - x_want) <= 4 * np.finfo(np.float64).eps * scale), "x_new"
    assert np.array_equal(xs[odd].cpu().numpy(), x), "x_old untouched"
    p_got = dp[1 - odd].cpu().numpy().astype(np.float64)
    assert np.all(np.abs(p_got - f32(direction)) <= np.spacing(np.abs(direction).astype(np.float32))), "p_new"
    assert np.array_equal(dp[odd].cpu().numpy(), p[odd].astype(np.float32)), "p_prev untouched"
    az, scale = apply_A(x_want, screen, pw)
    r_want = b - az
    r_got = from_padded(L, r32, n)
    assert np.abs(r_got - f32(r_want)).max() <= 1e-12 * scale.max() + np.spacing(np.float32(np.abs(r_want).max())), \
        "r32"
    assert float(scal[4].item()) == pytest.approx(float(np.sum(r_want ** 2)), rel=1e-9)
    assert np.array_equal(scal.cpu().numpy()[:4], [1.0, beta, alpha, 0.0]), "scalars untouched"


@pytest.mark.parametrize("n", (33, 65))
def test_fcg_launch_variants_are_bit_identical(L, n):
    """Every launch shape the autotuner may choose (register budgets, the
    cp.async-prefetching pass 2, planes per block) gives the same bits."""
    from mojo_poissonrecon_b200 import tune

    pw = 4.0
    screen, b, x, z, r, p = fcg_state(L, n, 99 + n)
    dz, dr = to_padded(L, z.astype(np.float32)), to_padded(L, r.astype(np.float32))
    ds, db = dev(screen), dev(b)
    ws = torch.empty(int(L.pb_fcg_workspace_size(n)), dtype=torch.uint8, device="cuda")

    def run():
        dp = [dev(a, torch.float32) for a in p]
        xs = [dev(x), torch.zeros((n, n, n), dtype=torch.float64, device="cuda")]
        scal = torch.zeros(8, dtype=torch.float64, device="cuda")
        scal[0] = 7.5
        flags = torch.tensor([0, 0, 1, 0], dtype=torch.int32, device="cuda")
        r32 = torch.zeros(geometry(L, n)[1], dtype=torch.float32, device="cuda")
        rin = dr.clone()
        s = stream()
        assert L.pb_fcg_direction_f64(dz.data_ptr(), dp[0].data_ptr(), dp[1].data_ptr(), rin.data_ptr(),
                                      ds.data_ptr(), n, pw, scal.data_ptr(), flags.data_ptr(), ws.data_ptr(),
                                      ws.numel(), s) == 0
        assert L.pb_fcg_update_f64(dz.data_ptr(), dp[0].data_ptr(), dp[1].data_ptr(), xs[0].data_ptr(),
                                   xs[1].data_ptr(), db.data_ptr(), ds.data_ptr(), r32.data_ptr(), n, pw,
                                   scal.data_ptr(), flags.data_ptr(), ws.data_ptr(), ws.numel(), s) == 0
        return [t.cpu() for t in (scal, xs[1], dp[1], r32)]

    L.pb_tune_clear()
    try:
        want = run()
        for param, value in [(tune.FCG_UPDATE_VARIANT, v) for v in (1, 2, 3, 4)] + \
                            [(tune.FCG_DIRECTION_VARIANT, v) for v in (1, 2)]:
            assert param in tune.SEARCHED
            assert L.pb_tune_set(param, n, value) == 0
            got = run()
            for a, b_ in zip(got, want):
                assert torch.equal(a, b_), (param, value)
            L.pb_tune_clear()
        # planes per block reshape the partial-sum trees: equal to rounding, not searched
        for param, value in ((tune.FCG_UPDATE_PLANES, 8), (tune.FCG_DIRECTION_PLANES, 12)):
            assert param not in tune.SEARCHED
            assert L.pb_tune_set(param, n, value) == 0
            got = run()
            for a, b_ in zip(got, want):
                assert torch.allclose(a.double(), b_.double(), rtol=1e-9, atol=1e-9 * float(b_.abs().max())), \
                    (param, value)
            L.pb_tune_clear()
    finally:
        L.pb_tune_clear()
