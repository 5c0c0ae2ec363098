"""Parity at the benchmarked sizes, against the CPU oracle (OpenMP build,
bit-identical to its serial build).

* Depth 8 (257^3), the benchmark's cloud: 1,000,000 torus samples (R 0.6,
  r 0.25, noise 0.002, normals scaled by a confidence U(0.5, 1.5), seed 1),
  confidence=True, point weight 4.
  - FP64 at a fixed 2 V-cycles: field, density, screen, rhs and the six octree
    arrays bit-identical; iso-value and residual norm within 1e-12 relative;
    the reconstructed mesh's faces identical and vertices within 1e-12.
  - FP32-refined to rel-res 1e-8 against the oracle solved to 1e-11: density,
    screen and rhs bit-identical (built before the solve), the field within
    REFINED_FIELD_TOL of the oracle's largest |field| (max norm), the iso-value
    within REFINED_ISO_TOL relative, and the mesh's face count within
    REFINED_FACES_TOL (relative) of the oracle's.
* Depth 10 (1025^3), 4,000,000 samples on 64 spheres: the refined field and
  mesh against the GPU FP64 solve to 1e-10 on the same grids.
* Depth 9 (513^3), 2,000,000 samples on a union of 64 spheres (seed 2): FP64
  at 1 V-cycle bit-identical to the oracle; the FP32-refined solve against the
  GPU's FP64 solve (bit-identical to the oracle cycle for cycle) run to 1e-11.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

REFINED_FIELD_TOL = 2e-6   # max |x_refined - x_oracle(1e-11)| / max |x_oracle|
REFINED_ISO_TOL = 1e-6     # relative
REFINED_FACES_TOL = 2e-3   # |F_refined - F_oracle| / F_oracle


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def torus(oracle):
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.torus(1_000_000, seed=1)
    keep = oracle.valid_rows(pts, nrm)
    unit, _, _ = oracle.normalize(pts[keep], 1.1)
    return pts, nrm, np.ascontiguousarray(unit), np.ascontiguousarray(nrm[keep])


@pytest.fixture(scope="module")
def torus_oracle_tight(oracle, torus):
    _, _, unit, n = torus
    return oracle.solve(unit, n, depth=8, confidence=True, point_weight=4.0, tol=1e-11, max_cycles=150,
                        threaded=True, octree=False)


def test_depth8_fp64_fixed_cycles_bit_exact(oracle, torus):
    import mojo_poissonrecon_b200 as mpr

    _, _, unit, n = torus
    got = mpr.solve_screened_poisson(unit, n, depth=8, confidence=True, point_weight=4.0, cycles=2)
    want = oracle.solve(unit, n, depth=8, confidence=True, point_weight=4.0, cycles=2, threaded=True)
    for k in ("field", "density", "screen", "rhs"):
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    for k in ("depth", "morton", "parent", "child_start", "child_count", "point_leaf"):
        assert np.array_equal(getattr(got.octree, k), getattr(want.octree, k)), k
    assert got.iso_value == pytest.approx(want.iso_value, rel=1e-12)
    assert got.residual_norm == pytest.approx(want.residual_norm, rel=1e-12)


def test_depth8_fp64_mesh_matches_oracle(oracle, torus):
    import mojo_poissonrecon_b200 as mpr

    pts, nrm, _, _ = torus
    got = mpr.reconstruct(pts, nrm, depth=8, confidence=True, point_weight=4.0, cycles=2)
    want = oracle.reconstruct(pts, nrm, depth=8, confidence=True, point_weight=4.0, cycles=2, threaded=True,
                              octree=False)
    assert got.faces.shape[0] > 100_000
    assert np.array_equal(got.faces, want.faces)
    assert np.allclose(got.vertices, want.vertices, rtol=0, atol=1e-12)
    assert np.allclose(got.density, want.density, rtol=0, atol=1e-12)
    assert got.iso_value == pytest.approx(want.iso_value, rel=1e-12)


def test_depth8_refined_within_stated_tolerance(oracle, torus, torus_oracle_tight):
    import mojo_poissonrecon_b200 as mpr

    _, _, unit, n = torus
    want = torus_oracle_tight
    assert want.relative_residual <= 1e-11
    got = mpr.solve_screened_poisson(unit, n, depth=8, confidence=True, point_weight=4.0,
                                     precision="fp32_refined", tol=1e-8)
    assert got.relative_residual <= 1e-8
    for k in ("density", "screen", "rhs"):
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    err = np.abs(got.field - want.field).max() / np.abs(want.field).max()
    assert err <= REFINED_FIELD_TOL, err
    assert got.iso_value == pytest.approx(want.iso_value, rel=REFINED_ISO_TOL)


def test_depth8_refined_mesh_close_to_oracle(oracle, torus, torus_oracle_tight):
    import mojo_poissonrecon_b200 as mpr

    pts, nrm, _, _ = torus
    got = mpr.reconstruct(pts, nrm, depth=8, confidence=True, point_weight=4.0, precision="fp32_refined",
                          tol=1e-8)
    sol = torus_oracle_tight
    want = oracle.extract(sol.field, sol.iso_value, sol.density, threaded=True)
    fo, fg = want.faces.shape[0], got.faces.shape[0]
    assert abs(fg - fo) <= REFINED_FACES_TOL * fo, (fg, fo)
    assert abs(got.vertices.shape[0] - want.vertices.shape[0]) <= REFINED_FACES_TOL * want.vertices.shape[0]


@pytest.fixture(scope="module")
def spheres9(oracle):
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.sphere_union(2_000_000, spheres=64, seed=2)
    keep = oracle.valid_rows(pts, nrm)
    unit, _, _ = oracle.normalize(pts[keep], 1.1)
    return np.ascontiguousarray(unit), np.ascontiguousarray(nrm[keep])


def test_depth9_fp64_one_cycle_bit_exact(oracle, spheres9):
    import mojo_poissonrecon_b200 as mpr

    unit, n = spheres9
    got = mpr.solve_screened_poisson(unit, n, depth=9, point_weight=4.0, cycles=1)
    want = oracle.solve(unit, n, depth=9, point_weight=4.0, cycles=1, threaded=True)
    for k in ("field", "density", "screen", "rhs"):
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
        setattr(want, k, None)  # 1 GB each: release as we go
    for k in ("depth", "morton", "parent", "child_start", "child_count", "point_leaf"):
        assert np.array_equal(getattr(got.octree, k), getattr(want.octree, k)), k
    assert got.iso_value == pytest.approx(want.iso_value, rel=1e-12)


def test_depth9_refined_against_tight_fp64(spheres9):
    import mojo_poissonrecon_b200 as mpr

    unit, n = spheres9
    dp, dn = torch.from_numpy(unit).cuda(), torch.from_numpy(n).cuda()
    got = mpr.solve_screened_poisson(dp, dn, depth=9, point_weight=4.0, precision="fp32_refined", tol=1e-8,
                                     device_out=True)
    assert got.relative_residual <= 1e-8
    want = mpr.solve_screened_poisson(dp, dn, depth=9, point_weight=4.0, precision="fp64", tol=1e-11,
                                      max_cycles=200, device_out=True)
    assert want.relative_residual <= 1e-11
    err = float((got.field - want.field).abs().max() / want.field.abs().max())
    assert err <= REFINED_FIELD_TOL, err
    assert got.iso_value == pytest.approx(want.iso_value, rel=REFINED_ISO_TOL)


def test_depth10_refined_against_tight_fp64():
    """Depth 10 (1025^3, the deep configuration's grid) with 4,000,000 samples on
    64 spheres: the FP32-refined field at rel-res 1e-8 against the FP64 solve to
    1e-10 on the same grids (the FP64 path is bit-identical to the oracle cycle
    for cycle at depths 8 and 9 above), and the refined reconstruction's mesh
    counts against the FP64 one's."""
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import core, solver32, workloads

    pts, nrm = workloads.sphere_union(4_000_000, spheres=64, seed=2)
    dp, dn = torch.from_numpy(pts).cuda(), torch.from_numpy(nrm).cuda()
    del pts, nrm
    ctx = core._Context()
    up, un, _, _ = core._prepare(ctx, dp, dn, 1.1)
    kw = dict(depth=10, point_weight=4.0, confidence=False, cycles=4, samples_per_node=1.5, max_cycles=400,
              octree=False)
    f32, _, _, st32, _ = core._solve_device(ctx, up, un, precision="fp32_refined", tol=1e-8, **kw)
    assert st32.relative_residual <= 1e-8
    solver32.clear_engines()
    f64, _, _, st64, _ = core._solve_device(ctx, up, un, precision="fp64", tol=1e-10, **kw)
    assert st64.relative_residual <= 1e-10
    err = float((f32 - f64).abs().max() / f64.abs().max())
    assert err <= REFINED_FIELD_TOL, err
    del f32, f64, up, un
    torch.cuda.empty_cache()
    a = mpr.reconstruct(dp, dn, depth=10, precision="fp32_refined", tol=1e-8, device_out=True)
    na, fa = a.vertices.shape[0], a.faces.shape[0]
    del a
    b = mpr.reconstruct(dp, dn, depth=10, precision="fp64", tol=1e-10, max_cycles=400, device_out=True)
    assert fa > 1_000_000
    assert abs(fa - b.faces.shape[0]) <= REFINED_FACES_TOL * b.faces.shape[0]
    assert abs(na - b.vertices.shape[0]) <= REFINED_FACES_TOL * b.vertices.shape[0]
