"""The FP32 preconditioner's Galerkin levels (csrc/mg27.cu, scaled level-0
transfers) against the CPU restatement in tests/mg_reference.py.

Tolerances (max norm, relative to the largest magnitude of the compared
quantity): Galerkin planes 3e-5 (FP32 products and sums over three
separable stages of 81 terms each, compounded over levels); weights and 1/diagonal 1e-5; packed FP16 couplings
exactly (the same FP32 operations, then rounding to FP16); a single sweep,
residual, restriction or prolongation 2e-6 to 4e-6 of the largest term,
evaluated on the GPU's own coefficients (FP32 planes, or the packed FP16
couplings) so only that kernel's rounding is measured; the 3^3 inverse (FP64) 1e-11;
whole cycles 1e-4."""

import numpy as np
import pytest

import mg_reference as mg
from padded import from_padded, ghosts_zero, to_padded

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mojo_poissonrecon_b200 import _native

    return _native.lib()


def shell_screen(n, seed):
    """Screening concentrated on a spherical shell, as splatting gives."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*(np.linspace(0, 1, n),) * 3, indexing="ij")
    r = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
    return np.where(np.abs(r - 0.3) < 1.5 / (n - 1), 5.0 + 20.0 * rng.random((n, n, n)), 0.0)


def gpu_hierarchy(n, screen):
    from mojo_poissonrecon_b200.solver32 import Hierarchy32

    h = Hierarchy32(n, torch.device("cuda"))
    h.setup(torch.from_numpy(screen).cuda(), 4.0)
    torch.cuda.synchronize()
    return h


def gpu_planes(L, lv):
    return np.stack([from_padded(L, lv.coef[k], lv.n) for k in range(14)])


def gpu_packed(lv):
    """The GPU's packed arrays of a level as (h0, h1, inv0, inv1) NumPy arrays."""
    n, pc = lv.n, (lv.n + 1) // 2
    h0, h1, i0, i1 = (t.cpu().numpy() for t in lv.packed)
    planes = lambda h: np.ascontiguousarray(np.moveaxis(h.reshape(n, n, pc, 32)[..., :26], -1, 0))
    assert not h0.reshape(n, n, pc, 32)[..., 26:].any() and not h1.reshape(n, n, pc, 32)[..., 26:].any()
    return (planes(h0), planes(h1), i0.reshape(n, n, pc), i1.reshape(n, n, pc))


def stream():
    return torch.cuda.current_stream().cuda_stream


def gpu_ops(L, h):
    """Operators and weights of the GPU hierarchy as FP64 sparse matrices."""
    ops, ws = [], []
    for lv in h.levels:
        if lv.coef is None:  # level 0 with the reference's 7-point operator
            ops.append(mg.operator7(from_padded(L, lv.D, lv.n)))
        elif lv.packed is not None:  # the rounded couplings the packed kernels apply
            ops.append(mg.packed_operator(*gpu_packed(lv), lv.n))
        else:
            ops.append(mg.from_planes(gpu_planes(L, lv), lv.n))
        ws.append(from_padded(L, lv.weights, lv.n).ravel())
    return ops, ws, [lv.n for lv in h.levels]


@pytest.mark.parametrize("n", [33, 65])
def test_galerkin_slabs_match_single_pass(L, n):
    """The separable product over slabs of one or three coarse planes (small
    workspaces) equals the single-slab product bit for bit: every node's
    arithmetic is the same whatever the slab; too small a workspace is an error."""
    from mojo_poissonrecon_b200 import _native

    h = gpu_hierarchy(n, shell_screen(n, 7))
    fine, coarse = h.levels[1], h.levels[2]
    fn, cn = fine.n, coarse.n
    full = coarse.coef.clone()
    one_plane = 27 * 4 * 3 * cn * (fn + cn)
    for nbytes in (one_plane, 27 * 4 * 7 * cn * (fn + cn) + 100):
        ws = torch.empty(nbytes // 4 + 1, dtype=torch.float32, device="cuda")
        out = torch.zeros_like(full)
        _native.check(L.pb_galerkin_f32(fine.coef.data_ptr(), fn, 0, fine.weights.data_ptr(), out.data_ptr(),
                                        ws.data_ptr(), nbytes, stream()), "galerkin slabs")
        torch.cuda.synchronize()
        assert torch.equal(out, full)
    ws = torch.empty(one_plane // 4, dtype=torch.float32, device="cuda")
    assert L.pb_galerkin_f32(fine.coef.data_ptr(), fn, 0, fine.weights.data_ptr(), full.data_ptr(), ws.data_ptr(),
                             one_plane - 4, stream()) != 0
    assert L.pb_galerkin_workspace_size(fn, 1) == 0 and L.pb_galerkin_workspace_size(fn, 0) >= one_plane


@pytest.mark.parametrize("n", [9, 17, 33, 65])
def test_galerkin_levels_match_restatement(L, n):
    screen = shell_screen(n, n)
    ops, ws, sizes = mg.hierarchy(screen, 4.0)
    h = gpu_hierarchy(n, screen)
    assert [lv.n for lv in h.levels] == sizes
    for l, lv in enumerate(h.levels):
        assert np.abs(from_padded(L, lv.weights, lv.n) - ws[l].reshape(lv.n, lv.n, lv.n)).max() <= 1e-5
        assert ghosts_zero(L, lv.weights, lv.n)
        if lv.coef is None:
            continue
        got, want = gpu_planes(L, lv), mg.planes(ops[l], lv.n)
        scale = np.abs(want).max()
        assert np.abs(got - want).max() <= 3e-5 * scale, (l, np.abs(got - want).max() / scale)
        inv = 1.0 / ops[l].diagonal().reshape(lv.n, lv.n, lv.n)
        assert np.abs(from_padded(L, lv.invD, lv.n) - inv).max() <= 1e-5 * np.abs(inv).max()
        for k in range(14):
            assert ghosts_zero(L, lv.coef[k], lv.n)


@pytest.mark.parametrize("n", [33, 65])
def test_pack27_matches_restatement(L, n):
    """Packed FP16 couplings and FP32 1/diagonal of level 1, exactly."""
    h = gpu_hierarchy(n, shell_screen(n, 2 * n))
    lv = h.levels[1]
    want = mg.pack(mg.from_planes(gpu_planes(L, lv), lv.n), lv.n)
    for got, w in zip(gpu_packed(lv), want):
        assert np.array_equal(got.view(np.uint16) if got.dtype == np.float16 else got.view(np.uint32),
                              w.view(np.uint16) if w.dtype == np.float16 else w.view(np.uint32))


@pytest.mark.parametrize("n", [33, 65, 129])
def test_relax27p_and_transfers(L, n):
    """One sweep (from a start and from zero) and the residual with the scaled
    restriction on a packed level (level 1), against the restated packed
    operator; the scaled prolongation on level 1."""
    h = gpu_hierarchy(n, shell_screen(n, 3 * n))
    lv, nxt = h.levels[1], h.levels[2]
    m, cm = lv.n, nxt.n
    A = mg.packed_operator(*gpu_packed(lv), m)
    s1 = from_padded(L, lv.weights, m).ravel()
    rng = np.random.default_rng(n)
    e = rng.normal(size=(m,) * 3).astype(np.float32).astype(np.float64)
    rhs = (rng.normal(size=(m,) * 3) * np.abs(A.diagonal()).max()).astype(np.float32).astype(np.float64)
    coarse = rng.normal(size=(cm,) * 3).astype(np.float32).astype(np.float64)
    lv.rhs.copy_(to_padded(L, rhs))
    e_in = to_padded(L, e)
    out = torch.zeros_like(e_in)
    terms = np.abs(A).sum(axis=1).max() * np.abs(e).max() + np.abs(rhs).max()
    dmin = A.diagonal().min()
    for zero in (False, True):
        assert L.pb_relax27p_f32(None if zero else e_in.data_ptr(), out.data_ptr(), lv.rhs.data_ptr(),
                                 *lv.packed_ptrs(), m, stream()) == 0, L.pb_last_error()
        want = mg.relax(A, e, rhs, m, zero=zero)
        # two dependent half-sweeps: an FP32 sum of 27 terms each, divided by the diagonal
        assert np.abs(from_padded(L, out, m) - want).max() <= 4e-6 * terms / dmin
        assert ghosts_zero(L, out, m)
    coarse_rhs = torch.zeros_like(nxt.rhs)
    assert L.pb_residual_restrict27p_f32(e_in.data_ptr(), lv.rhs.data_ptr(), *lv.packed_ptrs(),
                                         lv.weights.data_ptr(), m, lv.res.data_ptr(), coarse_rhs.data_ptr(),
                                         stream()) == 0
    want_c, want_r = mg.residual_restrict(A, s1, e, rhs, m)
    assert np.abs(from_padded(L, lv.res, m) - want_r).max() <= 2e-6 * terms
    assert np.abs(from_padded(L, coarse_rhs, cm) - want_c).max() <= 2e-6 * terms
    assert ghosts_zero(L, coarse_rhs, cm)
    fine = to_padded(L, e)
    assert L.pb_prolong_fac_f32(to_padded(L, coarse).data_ptr(), fine.data_ptr(), lv.weights.data_ptr(), m,
                                stream()) == 0
    want = mg.prolong(e, coarse, s1, m)
    assert np.abs(from_padded(L, fine, m) - want).max() <= 2e-6 * np.abs(want).max()
    assert ghosts_zero(L, fine, m)


def test_coarse_inverse(L):
    """The 3^3 level's inverse against a dense FP64 inverse of its GPU planes."""
    h = gpu_hierarchy(17, shell_screen(17, 1))
    A = mg.from_planes(gpu_planes(L, h.levels[-1]), 3).toarray()
    got = h.inverse.cpu().numpy().reshape(27, 27)
    assert got.dtype == np.float64
    want = np.linalg.inv(A)
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()


@pytest.mark.parametrize("n", [17, 33])
def test_coarse_block_cycle(L, n):
    """The single-block cycle over levels of side <= 17 against the restated cycle."""
    h = gpu_hierarchy(n, shell_screen(n, 5 * n))
    k = h.first_coarse
    ops, ws, sizes = gpu_ops(L, h)
    m = sizes[k]
    rhs = np.random.default_rng(n).normal(size=(m,) * 3).astype(np.float32).astype(np.float64)
    h.levels[k].rhs.copy_(to_padded(L, rhs))
    got = from_padded(L, h.v_cycle(k), m)
    want = mg.v_cycle(ops, ws, sizes, k, rhs, coarse_sweeps=h.coarse_sweeps)
    assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()


@pytest.mark.parametrize("n", [33, 65])
def test_full_cycle(L, n):
    """Level 0 (TMA sweeps, fused scaled transfers) down to 3^3 against the
    restated cycle on the GPU's own planes."""
    h = gpu_hierarchy(n, shell_screen(n, 11 * n))
    D0 = from_padded(L, h.levels[0].D, n)
    ops, ws, sizes = gpu_ops(L, h)
    rhs = (np.random.default_rng(n).normal(size=(n,) * 3) * D0.max()).astype(np.float32).astype(np.float64)
    h.levels[0].rhs.copy_(to_padded(L, rhs))
    got = from_padded(L, h.v_cycle(0), n)
    h.check_status()
    want = mg.v_cycle(ops, ws, sizes, 0, rhs, coarse_sweeps=h.coarse_sweeps)
    assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()


@pytest.mark.parametrize("n", [17, 65, 129])
def test_packed_level_tiled_variants_bit_identical(n):
    """The shared-memory staged packed sweep and residual (tuner variants) give
    the same bits as the gather kernels, from zero and from a previous iterate."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mojo_poissonrecon_b200 import _native, solver32, tune

    L = _native.lib()
    dev = torch.device("cuda")
    h = solver32.Hierarchy32(2 * n - 1, dev)
    rng = torch.Generator(device=dev).manual_seed(n)
    screen = torch.rand((2 * n - 1,) * 3, dtype=torch.float64, device=dev, generator=rng) * 3
    h.setup(screen, 4.0)
    lv = h.levels[1]
    assert lv.n == n and lv.packed is not None
    lv.rhs.copy_(torch.randn(lv.rhs.shape, device=dev, generator=rng) * (lv.invD != 0))
    lv.ea.copy_(torch.randn(lv.ea.shape, device=dev, generator=rng) * (lv.invD != 0))
    s = torch.cuda.current_stream().cuda_stream

    def sweep(zero):
        out = torch.zeros_like(lv.ea)
        assert L.pb_relax27p_f32(None if zero else lv.ea.data_ptr(), out.data_ptr(), lv.rhs.data_ptr(),
                                 *lv.packed_ptrs(), n, s) == 0
        return out

    def residual():
        res = torch.zeros_like(lv.ea)
        coarse = torch.zeros_like(h.levels[2].rhs)
        assert L.pb_residual_restrict27p_f32(lv.ea.data_ptr(), lv.rhs.data_ptr(), *lv.packed_ptrs(),
                                             lv.weights.data_ptr(), n, res.data_ptr(), coarse.data_ptr(), s) == 0
        return res, coarse

    L.pb_tune_clear()
    try:
        want = [sweep(False), sweep(True), *residual()]
        L.pb_tune_set(tune.RELAX27_VARIANT, n, 1)
        L.pb_tune_set(tune.RESIDUAL27_VARIANT, n, 1)
        got = [sweep(False), sweep(True), *residual()]
        for a, b in zip(got, want):
            assert torch.equal(a, b)
    finally:
        L.pb_tune_clear()
