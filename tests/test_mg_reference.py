"""CPU checks of the preconditioner's restatement (tests/mg_reference.py):
its storage round trip, and the convergence property that motivates the
Galerkin levels, on a depth-5 sphere assembled by the oracle."""

import numpy as np
import pytest

import mg_reference as mg


@pytest.fixture(scope="module")
def sphere_system(oracle):
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.sphere(3000, seed=0)
    unit, _, _ = oracle.normalize(pts, 1.1)
    _, screen, rhs = oracle.splat_and_assemble(unit, nrm, 5, 4.0, False, 1.5)
    return screen, rhs


def test_planes_round_trip():
    rng = np.random.default_rng(0)
    screen = rng.random((9, 9, 9)) * (rng.random((9, 9, 9)) < 0.3)
    ops, ws, sizes = mg.hierarchy(screen, 4.0)
    for A, n in zip(ops[1:], sizes[1:]):
        assert abs(mg.from_planes(mg.planes(A, n), n) - A).max() <= 1e-12 * abs(A).max()
        assert abs(A - A.T).max() <= 1e-12 * abs(A).max()
    for s in ws:
        assert s.min() >= 0.0 and s.max() <= 1.0


@pytest.mark.parametrize("n", [9, 17])
def test_separable_galerkin_equals_direct_product(n):
    """The x, y, z stages of the 27-point Galerkin product (as the GPU runs
    them) equal the direct sparse product P_s^T A P_s / 8, boundary rows
    included, for a realistic 27-point level (the Galerkin level below a
    7-point one with shell screening) and for a random symmetric one."""
    rng = np.random.default_rng(n)
    fine = 2 * n - 1
    screen = rng.random((fine, fine, fine)) * (rng.random((fine, fine, fine)) < 0.2) * 50.0
    ops, ws, sizes = mg.hierarchy(screen, 4.0)
    A, s = ops[1], ws[1]
    assert sizes[1] == n
    cn = (n + 1) // 2
    want = mg.planes(mg.galerkin(A, s, n), cn)
    got = mg.galerkin_separable(A, s, n)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    R = mg.from_planes(rng.normal(size=(14, n, n, n)) * (np.arange(14) > 0)[:, None, None, None], n)
    R = R + R.T
    s2 = rng.random(n ** 3)
    want = mg.planes(mg.galerkin(R, s2, n), cn)
    assert np.abs(mg.galerkin_separable(R, s2, n) - want).max() <= 1e-12 * np.abs(want).max()


def _reference_factors(oracle, screen, rhs, cycles):
    """Residual ratios of the reference's rediscretised V(3,3) cycle (oracle)."""
    L = oracle.lib()
    a = lambda v: int(v.ctypes.data)
    screens = [screen]
    while screens[-1].shape[0] > 3:
        screens.append(oracle.restrict(screens[-1]) * 4.0)
    sol = [np.full_like(s, 0.5) for s in screens]
    rhs_levels = [np.zeros_like(s) for s in screens]
    res = [np.empty_like(s) for s in screens]
    rhs_levels[0][...] = rhs
    n = rhs.shape[0]
    norms = [L.mpr_residual_f64(a(sol[0]), a(rhs), a(screen), a(res[0]), n, 4.0)]
    for _ in range(cycles):
        oracle._v_cycle(0, sol, rhs_levels, screens, res, 4.0, 3, 3, L)
        norms.append(L.mpr_residual_f64(a(sol[0]), a(rhs), a(screen), a(res[0]), n, 4.0))
    return [norms[k + 1] / norms[k] for k in range(cycles)]


def test_galerkin_cycle_contracts(oracle, sphere_system):
    """x += V(b - A x) with the restated cycle gains at least 10x per cycle;
    the reference's rediscretised V(3,3) cycle settles at under 5x per cycle on the
    same system (which is why the refined solvers use the Galerkin levels)."""
    screen, rhs = sphere_system
    n = screen.shape[0]
    ops, ws, sizes = mg.hierarchy(screen, 4.0)
    A, b = ops[0], rhs.ravel()
    x = np.full(n ** 3, 0.5)
    norms = [np.linalg.norm(b - A @ x)]
    for _ in range(4):
        x = x + mg.v_cycle(ops, ws, sizes, 0, (b - A @ x).reshape(n, n, n)).ravel()
        norms.append(np.linalg.norm(b - A @ x))
    factors = [norms[k + 1] / norms[k] for k in range(len(norms) - 1)]
    assert max(factors[1:]) <= 0.1, factors
    reference = _reference_factors(oracle, screen, rhs, 4)
    assert reference[-1] >= 0.2, reference


def test_operator7_is_the_references(oracle, sphere_system):
    screen, _ = sphere_system
    n = screen.shape[0]
    A = mg.operator7(mg.level0_diagonal(screen, 4.0))
    x = np.random.default_rng(1).normal(size=(n, n, n))
    zero, res = np.zeros_like(x), np.empty_like(x)
    oracle.lib().mpr_residual_f64(int(x.ctypes.data), int(zero.ctypes.data), int(screen.ctypes.data),
                                  int(res.ctypes.data), n, 4.0)
    assert np.abs(A @ x.ravel() + res.ravel()).max() <= 1e-12 * np.abs(res).max()
