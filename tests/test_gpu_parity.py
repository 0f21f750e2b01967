"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

Golden data: tests/golden/*.npz from the reference's own code (make_golden.py).  When
oracle/_ref is present, the 1000-step configuration also runs live for an element-wise
comparison of every population.
"""
import os

import numpy as np
import pytest

from gpu_helpers import GpuSim, l2rel, rel
from oracle.bindings import SphereCase
from periodicshiftlbm_b200 import debug_cells

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="module")
def cells():
    return load("cell_functions.npz")


def test_collision_kernel_matches_reference(cells):
    F = cells["f_in"]
    for p, (nu, cs) in enumerate(cells["collision_params"]):
        args = np.tile(np.array([nu, cs, 0, 0], dtype=np.float32), (F.shape[0], 1))
        got = debug_cells(0, 0, F, args)
        # FMA contraction and the central-moment form of |Pi_neq|: FP32 rounding only
        assert rel(got, cells["collision_out"][p]) < 5e-6, (nu, cs, rel(got, cells["collision_out"][p]))


def test_rescale_kernel_matches_reference(cells):
    F = cells["f_in"]
    args = np.zeros((F.shape[0], 4), dtype=np.float32)
    assert rel(debug_cells(1, 1, F, args), cells["rescale_c2f"]) < 5e-6
    assert rel(debug_cells(1, 0, F, args), cells["rescale_f2c"]) < 5e-6


def test_boundary_kernels_bitwise_equal_reference(cells):
    """The generated boundary code evaluates the reference's operations in the reference's
    order with explicit round-to-nearest intrinsics: identical inputs give identical bits."""
    F = cells["f_in"]
    n = F.shape[0]
    for a, nrm in enumerate(cells["bc_normals"]):
        idx = (int(nrm[0]) + 1) * 9 + (int(nrm[1]) + 1) * 3 + (int(nrm[2]) + 1)
        rho, u = cells["bc_rho"][a], cells["bc_u"][a]
        args = np.concatenate([rho[:, None], u], axis=1).astype(np.float32)
        assert np.array_equal(debug_cells(2, idx, F, args), cells["mbbc_out"][a]), tuple(nrm)
        args_r = np.concatenate([np.ones((n, 1), np.float32), u], axis=1)
        assert np.array_equal(debug_cells(3, idx, F, args_r)[:, 0], cells["restore_rho_out"][a])
        args_u = np.concatenate([rho[:, None], np.zeros((n, 3), np.float32)], axis=1)
        assert np.array_equal(debug_cells(4, idx, F, args_u)[:, :3], cells["restore_u_out"][a])
        args_ru = np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1))
        assert np.array_equal(debug_cells(5, idx, F, args_ru)[:, :4], cells["restore_rho_u_out"][a])
        assert np.array_equal(debug_cells(6, idx, F, np.zeros((n, 4), np.float32)), cells["mirror_out"][a])


def test_forced_collision_matches_oracle(orc, cells):
    F = cells["f_in"][:16]
    args = np.tile(np.array([0.01, 0.1, 1e-4, -2e-4], dtype=np.float32), (F.shape[0], 1))
    got = debug_cells(7, 0, F, args)
    want = np.stack([orc.collision(f, 0.01, 0.1, force=(1e-4, -2e-4, 0.0)) for f in F])
    assert rel(got, want) < 5e-6


CASES = {
    "tiny_mirror": SphereCase(nx=12, ny=8, nz=8, sphere=(4.0, 4.0, 4.0), radius=1.5, nu=0.02),
    "small_velwall_les": SphereCase(nx=24, ny=16, nz=16, sphere=(8.0, 8.0, 8.0), radius=3.0, nu=0.001,
                                    smagorinsky=0.1, wall_mode=1),
    "small_refined_les": SphereCase(nx=32, ny=16, nz=16, sphere=(14.0, 8.0, 8.0), radius=2.5, nu=0.005,
                                    smagorinsky=0.1, refine=((8, 4, 4), (20, 12, 12))),
    "config1_1000": SphereCase(),
}


def test_start_state_matches_oracle(orc):
    c = CASES["small_refined_les"]
    gpu = GpuSim(c)
    cpu = orc.sim(c)
    for lev in range(2):
        assert rel(gpu.populations(lev), cpu.populations(lev)) < 1e-6
    gpu.close()


def check_against_golden(sim, name, tol):
    g = load(f"run_{name}.npz")
    worst = 0.0
    for lev in range(sim.levels):
        f = sim.populations(lev)
        assert np.array_equal(sim.shifts(lev), g[f"shifts_{lev}"]), "periodic shifts are bit-exact"
        assert rel(f.astype(np.float64).sum(axis=1), g[f"checksum_{lev}"]) < 2e-6
        if f"f_{lev}" in g:
            r = rel(f, g[f"f_{lev}"])
        else:
            r = rel(f[:, g[f"sample_idx_{lev}"]], g[f"sample_f_{lev}"])
        worst = max(worst, r)
        assert r < tol, (name, lev, r)
    d = sim.drag()
    # the reference sums the per-cell momentum exchange in FP32 (cancelling terms), the
    # library in FP64
    assert abs(d - float(g["drag"])) <= 1e-4 * abs(float(g["drag"])), (d, float(g["drag"]))
    return worst


@pytest.mark.parametrize("name", ["tiny_mirror", "small_velwall_les", "small_refined_les"])
def test_gpu_runs_match_reference(name):
    g = load(f"run_{name}.npz")
    sim = GpuSim(CASES[name])
    sim.run(int(g["steps"]))
    check_against_golden(sim, name, tol=1e-5)
    sim.close()


def test_config1_1000_steps_matches_reference(ref):
    """Config 1 (128x64x64 sphere, Re=100), 1000 steps: every population of the CUDA path
    within 1e-5 relative of the reference's own update (run live on the host)."""
    c = CASES["config1_1000"]
    sim = GpuSim(c)
    sim.run(1000)
    check_against_golden(sim, "config1_1000", tol=1e-5)
    r = ref.sim(c)
    r.run(1000)
    fg, fr = sim.populations(), r.populations()
    assert np.array_equal(sim.shifts(), r.shifts())
    max_rel, l2 = rel(fg, fr), l2rel(fg, fr)
    print(f"config1 1000 steps: max rel {max_rel:.3e}, L2 rel {l2:.3e}, drag gpu {sim.drag():.7g} ref {r.drag():.7g}")
    assert l2 < 1e-6
    assert max_rel < 1e-5
    sim.close()


def test_three_levels_match_reference(ref):
    """Three refinement levels through psl_update_grid's recursion against the reference's
    own code: shifts exact, populations of every level within FP32 rounding."""
    c = SphereCase(nx=32, ny=24, nz=24, sphere=(13.0, 12.0, 12.0), radius=2.5, nu=0.004, smagorinsky=0.1,
                   refine=((6, 6, 6), (22, 18, 18)), refine2=((8, 6, 6), (24, 18, 18)))
    g = GpuSim(c)
    r = ref.sim(c)
    assert g.levels == 3
    g.run(10)
    r.run(10)
    for lev in range(3):
        assert np.array_equal(g.shifts(lev), r.shifts(lev)), lev
        assert rel(g.populations(lev), r.populations(lev)) < 1e-5, lev
    assert abs(g.drag() - r.drag()) <= 1e-4 * abs(r.drag())
    g.close()


def test_config2_full_size_matches_reference(ref):
    """The 512x256x256 case with its 256x192x192 refined block (Re = 1e5, Smagorinsky),
    full size, two coarse steps (two coarse updates, four fine updates, two transfers):
    every one of the 1.2e9 populations of the CUDA path within 1e-5 relative of the
    reference's own update run on the host, shifts exact."""
    from periodicshiftlbm_b200.cases import config2

    c2 = config2()
    case = SphereCase(nx=c2.nx, ny=c2.ny, nz=c2.nz, sphere=tuple(c2.sphere), radius=c2.radius, u_in=c2.u_in,
                      nu=c2.nu, smagorinsky=c2.smagorinsky, refine=c2.refine)
    sim = GpuSim(case)
    sim.run(2)
    r = ref.sim(case)
    r.run(2)
    for lev in range(2):
        assert np.array_equal(sim.shifts(lev), r.shifts(lev)), lev
        fg, fr = sim.populations(lev), r.populations(lev)
        assert fg.shape == fr.shape
        worst = max(rel(fg[q], fr[q]) for q in range(27))  # row by row: bounded host memory
        print(f"config2 level {lev}: max rel {worst:.3e} over {fg.size} populations")
        assert worst < 1e-5, (lev, worst)
        del fg, fr
    assert abs(sim.drag() - r.drag()) <= 1e-4 * abs(r.drag())
    sim.close()


def test_fill_coarse_from_fine_matches_reference(ref):
    """psl_fill_coarse_grid_from_fine against the reference's fillCoarseGridFromFine after the
    same 2-level run: the coarse level within FP32 rounding, cells outside the block and the
    fine level untouched."""
    from periodicshiftlbm_b200 import fillCoarseGridFromFine

    c = CASES["small_refined_les"]
    sim, r = GpuSim(c), ref.sim(c)
    sim.run(6)
    r.run(6)
    before_c, before_f = sim.populations(0), sim.populations(1)
    fillCoarseGridFromFine(sim.grids[0], sim.grids[1])
    r.fill_coarse_from_fine(0)
    fg = sim.populations(0)
    (i0, j0, k0), (i1, j1, k1) = c.refine
    inside = np.zeros((c.nz, c.ny, c.nx), dtype=bool)
    inside[k0 + 1:k1 - 1, j0 + 1:j1 - 1, i0 + 1:i1 - 1] = True
    inside = inside.ravel()
    assert rel(fg, r.populations(0)) < 1e-5
    assert np.array_equal(fg[:, ~inside], before_c[:, ~inside])
    assert not np.array_equal(fg[:, inside], before_c[:, inside])
    assert np.array_equal(sim.populations(1), before_f)
    assert sim.grids[0].health() == 0
    sim.close()
