"""Pin the CPU oracle (oracle/psl_oracle.cpp) against the reference's own code.

Golden fixtures in tests/golden/ come from the reference headers compiled unmodified for
the host (tests/golden/make_golden.py); when oracle/_ref is built, the live comparisons
run too.  No GPU needed.
"""
import os

import numpy as np
import pytest

from oracle.bindings import ALL_NORMALS, SphereCase

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)))


@pytest.fixture(scope="module")
def cells():
    return load("cell_functions.npz")


def test_collision_matches_reference(orc, cells):
    F = cells["f_in"]
    for p, (nu, cs) in enumerate(cells["collision_params"]):
        got = np.stack([orc.collision(f, float(nu), float(cs)) for f in F])
        # FP32 rounding-order differences only (loops vs the reference's named formulas)
        assert rel(got, cells["collision_out"][p]) < 3e-6, (nu, cs)


def test_rescale_matches_reference(orc, cells):
    F = cells["f_in"]
    assert rel(np.stack([orc.rescale(f, True) for f in F]), cells["rescale_c2f"]) < 3e-6
    assert rel(np.stack([orc.rescale(f, False) for f in F]), cells["rescale_f2c"]) < 3e-6


def test_boundary_conditions_match_reference(orc, cells):
    F = cells["f_in"]
    for a, nrm in enumerate(cells["bc_normals"]):
        nrm = tuple(int(v) for v in nrm)
        for i in range(F.shape[0]):
            rho = float(cells["bc_rho"][a, i])
            u = [float(v) for v in cells["bc_u"][a, i]]
            got = orc.mbbc(nrm, rho, *u, F[i])
            # unknown populations are differences of O(1) sums: absolute FP32 tolerance
            assert np.max(np.abs(got - cells["mbbc_out"][a, i])) < 2e-7, nrm
            assert abs(orc.restore_rho(nrm, *u, F[i]) - cells["restore_rho_out"][a, i]) < 2e-7
            assert np.max(np.abs(orc.restore_u(nrm, rho, F[i]) - cells["restore_u_out"][a, i])) < 2e-7
            assert np.max(np.abs(orc.restore_rho_u(nrm, F[i]) - cells["restore_rho_u_out"][a, i])) < 2e-7
            assert np.array_equal(orc.mirror(nrm, F[i]), cells["mirror_out"][a, i])


def test_bounceback_matches_reference(orc, cells):
    F = cells["f_in"]
    assert np.array_equal(np.stack([orc.bounceback(f) for f in F]), cells["bounceback_out"])
    u = [float(v) for v in cells["moving_bb_u"]]
    got = np.stack([orc.moving_bounceback(f, *u) for f in F])
    assert np.max(np.abs(got - cells["moving_bb_out"])) < 1e-8


def test_streaming_shifts_bit_exact(orc, cells):
    for dims, seq in zip(cells["stream_dims"], cells["stream_shifts"]):
        s = np.zeros(27, dtype=np.int32)
        for expect in seq:
            s = orc.streaming(tuple(int(v) for v in dims), s)
            assert np.array_equal(s, expect), dims


CASES = {
    "tiny_mirror": SphereCase(nx=12, ny=8, nz=8, sphere=(4.0, 4.0, 4.0), radius=1.5, nu=0.02),
    "small_velwall_les": SphereCase(nx=24, ny=16, nz=16, sphere=(8.0, 8.0, 8.0), radius=3.0, nu=0.001,
                                    smagorinsky=0.1, wall_mode=1),
    "small_refined_les": SphereCase(nx=32, ny=16, nz=16, sphere=(14.0, 8.0, 8.0), radius=2.5, nu=0.005,
                                    smagorinsky=0.1, refine=((8, 4, 4), (20, 12, 12))),
    "config1_1000": SphereCase(),
}


def check_run_against_golden(sim, name, tol_sample, tol_checksum=2e-6, tol_drag=1e-4):
    g = load(f"run_{name}.npz")
    for lev in range(sim.levels):
        f = sim.populations(lev)
        assert np.array_equal(sim.shifts(lev), g[f"shifts_{lev}"])
        cs = f.astype(np.float64).sum(axis=1)
        assert rel(cs, g[f"checksum_{lev}"]) < tol_checksum, (name, lev)
        if f"f_{lev}" in g:
            assert rel(f, g[f"f_{lev}"]) < tol_sample, (name, lev, rel(f, g[f"f_{lev}"]))
        else:
            idx = g[f"sample_idx_{lev}"]
            assert rel(f[:, idx], g[f"sample_f_{lev}"]) < tol_sample, (name, lev, rel(f[:, idx], g[f"sample_f_{lev}"]))
    # the reference reduces the per-cell momentum exchange in FP32 with cancelling terms
    assert abs(sim.drag() - float(g["drag"])) <= tol_drag * abs(float(g["drag"])), (sim.drag(), float(g["drag"]))


@pytest.mark.parametrize("name", ["tiny_mirror", "small_velwall_les", "small_refined_les"])
def test_oracle_runs_match_reference(orc, name):
    g = load(f"run_{name}.npz")
    sim = orc.sim(CASES[name])
    sim.run(int(g["steps"]))
    check_run_against_golden(sim, name, tol_sample=1e-5)


def test_oracle_config1_1000_steps_matches_reference(orc):
    """Config 1 (128x64x64, Re=100), 1000 steps: the oracle restatement stays within
    1e-5 relative of the reference on every sampled population."""
    sim = orc.sim(CASES["config1_1000"])
    sim.run(1000)
    check_run_against_golden(sim, "config1_1000", tol_sample=1e-5)


def test_double_oracle_tracks_float(orc):
    """The FP64 oracle (used for the reduced-precision forms) agrees with FP32 to FP32
    rounding on a short run."""
    c = CASES["small_velwall_les"]
    a = orc.sim(c)
    b = orc.sim(c, double=True)
    a.run(50)
    b.run(50)
    fa, fb = a.populations(), b.populations()
    assert fb.dtype == np.float64
    assert rel(fa, fb) < 2e-5


def test_live_reference_random_states(ref, orc):
    """Beyond the fixtures: random near-equilibrium states through every boundary normal."""
    rng = np.random.default_rng(99)
    for _ in range(10):
        u = rng.uniform(-0.06, 0.06, 3)
        f = (ref.feq(1.0, *u) * (1 + rng.uniform(-0.03, 0.03, 27))).astype(np.float32)
        assert rel(orc.collision(f, 0.01, 0.13), ref.collision(f, 0.01, 0.13)) < 3e-6
        for nrm in ALL_NORMALS:
            uu = rng.uniform(-0.05, 0.05, 3)
            assert np.max(np.abs(orc.mbbc(nrm, 1.0, *uu, f) - ref.mbbc(nrm, 1.0, *uu, f))) < 2e-7
            assert np.array_equal(orc.mirror(nrm, f), ref.mirror(nrm, f))


THREE_LEVELS = SphereCase(nx=32, ny=24, nz=24, sphere=(13.0, 12.0, 12.0), radius=2.5, nu=0.004, smagorinsky=0.1,
                          refine=((6, 6, 6), (22, 18, 18)), refine2=((8, 6, 6), (24, 18, 18)))


def test_three_levels_oracle_matches_reference(ref, orc):
    """The updateGrid recursion over three levels (flowAroundSphereMainSingle.cu:158-167):
    the restatement against the reference's own code, every level."""
    a = ref.sim(THREE_LEVELS)
    b = orc.sim(THREE_LEVELS)
    a.run(6)
    b.run(6)
    for lev in range(3):
        assert np.array_equal(a.shifts(lev), b.shifts(lev)), lev
        fa, fb = a.populations(lev), b.populations(lev)
        assert np.max(np.abs(fa - fb) / np.abs(fa)) < 1e-5, lev
    assert abs(a.drag() - b.drag()) <= 1e-4 * abs(a.drag())


def _block_mask(case):
    """Cells of the coarse box [iS+1, iE-1) x [jS+1, jE-1) x [kS+1, kE-1) (logical order)."""
    (i0, j0, k0), (i1, j1, k1) = case.refine
    m = np.zeros((case.nz, case.ny, case.nx), dtype=bool)
    m[k0 + 1:k1 - 1, j0 + 1:j1 - 1, i0 + 1:i1 - 1] = True
    return m.ravel()


def test_fill_coarse_from_fine_oracle_matches_reference(ref, orc):
    """fillCoarseGridFromFine (gridRefinementFunctions.h:528-535): after a 2-level run both
    checkers overwrite the coarse cells inside the block with the restricted fine state; the
    oracle's restatement stays within FP32 rounding of the reference and leaves every other
    coarse cell and the fine grid untouched."""
    c = CASES["small_refined_les"]
    a, b = ref.sim(c), orc.sim(c)
    a.run(6)
    b.run(6)
    before_c, before_f = b.populations(0), b.populations(1)
    a.fill_coarse_from_fine(0)
    b.fill_coarse_from_fine(0)
    fa, fb = a.populations(0), b.populations(0)
    inside = _block_mask(c)
    assert rel(fb, fa) < 1e-5
    assert np.array_equal(fb[:, ~inside], before_c[:, ~inside])
    assert not np.array_equal(fb[:, inside], before_c[:, inside])
    assert np.array_equal(b.populations(1), before_f)


def test_per_cell_smagorinsky_hook_field_equals_reference(ref):
    """The library's per-cell Smagorinsky field of the outlet-sponge case holds exactly the
    values the reference's getSmagorinskyConstant hook returns (coarse and fine grid)."""
    from periodicshiftlbm_b200.cases import SphereConfig, sponge_smagorinsky

    case = SphereCase(nx=40, ny=12, nz=10, sphere=(10.0, 6.0, 5.0), radius=2.0, nu=0.004, smagorinsky=0.1,
                      cs_mode=1, refine=((4, 2, 2), (16, 10, 8)))
    cfg = SphereConfig(name="t", nx=case.nx, ny=case.ny, nz=case.nz, sphere=case.sphere, radius=case.radius,
                       u_in=case.u_in, nu=case.nu, smagorinsky=case.smagorinsky, refine=case.refine, cs_mode=1)
    coarse = cfg.infos()[0]
    want = ref.smagorinsky_constants(case, 0, case.nx, case.ny, case.nz)
    got = sponge_smagorinsky(coarse, case.smagorinsky)
    assert np.array_equal(got, want)
    assert want.max() > 3.9 * case.smagorinsky and want.min() == np.float32(case.smagorinsky)
    fine = cfg.infos()[1]
    assert np.all(ref.smagorinsky_constants(case, 1, fine.cellCountX, fine.cellCountY, fine.cellCountZ)
                  == np.float32(case.smagorinsky))


def test_oracle_per_cell_smagorinsky_matches_reference(ref, orc):
    """The oracle restatement's per-cell hook against the reference run: a refined LES case
    with the outlet sponge, 40 steps."""
    case = SphereCase(nx=32, ny=16, nz=16, sphere=(12.0, 8.0, 8.0), radius=2.5, nu=0.002, smagorinsky=0.15,
                      cs_mode=1, refine=((6, 4, 4), (18, 12, 12)))
    r = ref.sim(case)
    o = orc.sim(case)
    r.run(40)
    o.run(40)
    for lev in range(2):
        a, b = o.populations(lev), r.populations(lev)
        assert np.max(np.abs(a.astype(np.float64) - b) / np.abs(b)) < 1e-5, lev
    # the sponge changes the solution: the uniform-constant run differs
    u = orc.sim(SphereCase(**{**case.__dict__, "cs_mode": 0}))
    u.run(40)
    assert np.max(np.abs(u.populations(0).astype(np.float64) - r.populations(0))) > 1e-7
    r.close()
    o.close()
    u.close()
