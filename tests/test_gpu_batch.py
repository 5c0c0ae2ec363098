"""Batched solves (one grouped launch per solver step across uneven clouds)
against the single-cloud path, cloud by cloud.

The batch runs the same kernels on the same data in the same order for every
cloud, so each field, iteration count and residual must be bit-identical to
the single-cloud RefinedEngine's, and each mesh of reconstruct_many identical
to core.reconstruct of that cloud alone (precision "fp32_refined", tol 1e-8)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def uneven_clouds(seed=21):
    from mojo_poissonrecon_b200 import workloads

    rng = np.random.default_rng(seed)
    out = []
    for depth, count in ((8, 60_000), (5, 3_000), (7, 40_000), (6, 12_000), (5, 800), (8, 150_000)):
        if rng.uniform() < 0.5:
            p, n = workloads.ellipsoid(count, rng)
        else:
            p, n = workloads.torus(count, major=0.55, minor=0.2, noise=0.0, confidence=None, rng=rng)
        out.append((p, n, depth))
    return out


def prepared_systems(clouds):
    """Per cloud: (rhs, screen) on the device, as core.reconstruct builds them."""
    from mojo_poissonrecon_b200 import core

    ctx = core._Context()
    systems = []
    for p, n, d in clouds:
        dp, dn, count, _ = core._prepare(ctx, core._to_device(p, ctx.device), core._to_device(n, ctx.device), 1.1)
        grids, _ = core._splat_assemble(ctx, dp, dn, d, 4.0, False, 1.5)
        systems.append((grids["rhs"], grids["screen"]))
    return systems


def test_batch_solver_bit_identical_to_single_engine():
    from mojo_poissonrecon_b200 import _native, batch, solver32

    clouds = uneven_clouds()
    systems = prepared_systems(clouds)
    solver = batch.BatchSolver([s[0].shape[0] for s in systems])
    fields, stats = solver.solve([s[0] for s in systems], [s[1] for s in systems], 4.0, tol=1e-8)
    for (rhs, screen), field, st in zip(systems, fields, stats):
        want, wst = solver32.solve_refined(rhs, screen, 4.0, _native.Workspace(rhs.device), tol=1e-8,
                                           max_cycles=200)
        assert st.cycles == wst.cycles
        assert st.residual_norm == wst.residual_norm
        assert st.rhs_norm == wst.rhs_norm
        assert torch.equal(field, want)
        assert st.residual_norm <= 1e-8 * st.rhs_norm


def test_batch_solver_repeatable_and_converged_clouds_frozen():
    """Solving twice gives the same bits; clouds that converge early keep the
    iterate they converged with while the others iterate on."""
    from mojo_poissonrecon_b200 import batch

    clouds = uneven_clouds(seed=5)[:4]
    systems = prepared_systems(clouds)
    solver = batch.BatchSolver([s[0].shape[0] for s in systems])
    a, sa = solver.solve([s[0] for s in systems], [s[1] for s in systems], 4.0, tol=1e-8)
    b, sb = solver.solve([s[0] for s in systems], [s[1] for s in systems], 4.0, tol=1e-8)
    for x, y, s1, s2 in zip(a, b, sa, sb):
        assert torch.equal(x, y) and s1.cycles == s2.cycles
    assert len({s.cycles for s in sa}) >= 1
    # a loose tolerance stops every cloud earlier, each at its own count
    c, sc = solver.solve([s[0] for s in systems], [s[1] for s in systems], 4.0, tol=1e-4)
    for s_tight, s_loose in zip(sa, sc):
        assert s_loose.cycles <= s_tight.cycles
        assert s_loose.residual_norm <= 1e-4 * s_loose.rhs_norm


def test_reconstruct_many_matches_single_reconstructions():
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import batch

    clouds = uneven_clouds(seed=9)
    pts, nrm = clouds[1][0].copy(), clouds[1][1].copy()
    nrm[:] = 0.0  # every row invalid: an empty mesh
    clouds.append((pts, nrm, 6))
    clouds.append((clouds[0][0][:5000], clouds[0][1][:5000], 4))  # below the batched solver: single path
    meshes = batch.reconstruct_many(clouds, tol=1e-8)
    assert len(meshes) == len(clouds)
    for (p, n, d), mesh in zip(clouds, meshes):
        want = mpr.reconstruct(p, n, depth=d, precision="fp32_refined", tol=1e-8)
        assert np.array_equal(mesh.vertices, want.vertices)
        assert np.array_equal(mesh.faces, want.faces)
        assert np.array_equal(mesh.density, want.density)
        assert mesh.iso_value == want.iso_value
        assert mesh.residual_norm == want.residual_norm
    assert meshes[-2].is_empty


def test_reconstruct_many_in_waves_matches_one_wave():
    from mojo_poissonrecon_b200 import batch

    clouds = uneven_clouds(seed=13)[:5]
    one = batch.reconstruct_many(clouds, tol=1e-8)
    many = batch.reconstruct_many(clouds, tol=1e-8, budget_bytes=1)  # every cloud its own wave
    for a, b in zip(one, many):
        assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.faces, b.faces)


def test_batch_with_a_depth9_cloud_matches_single_reconstructions():
    """A 513^3 cloud in a batch beside smaller ones: meshes identical to
    core.reconstruct alone (whose depth-9 engine runs lean)."""
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import batch, workloads

    rng = np.random.default_rng(29)
    clouds = []
    for depth, count in ((9, 120_000), (6, 20_000), (8, 60_000)):
        p, n = workloads.torus(count, major=0.5, minor=0.2, noise=0.0, confidence=None, rng=rng)
        clouds.append((p, n, depth))
    meshes = batch.reconstruct_many(clouds, tol=1e-8)
    for (p, n, d), mesh in zip(clouds, meshes):
        want = mpr.reconstruct(p, n, depth=d, precision="fp32_refined", tol=1e-8)
        assert np.array_equal(mesh.vertices, want.vertices) and np.array_equal(mesh.faces, want.faces), d
        assert mesh.residual_norm == want.residual_norm
