"""The FP64 oracle form and the reduced-precision storage forms on the GPU.

* FP64 storage with FP64 arithmetic (the runs the 16-bit forms are measured against)
  matches the CPU oracle's double-precision run: single level and two levels.
* The 16-bit shifted forms (f - w in FP16 / BF16, FP32 arithmetic) run through the
  coarse/fine transfer and stay close to the FP64 run; FP32 stays closer still.
* The FP64 macroscopic export agrees with moments taken from the exported populations.
"""
import numpy as np
import pytest

from gpu_helpers import GpuSim, l2rel, rel
from oracle.bindings import SphereCase
from periodicshiftlbm_b200.precision import speed_error, updated_cells

pytestmark = pytest.mark.gpu

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1])
CZ = np.array([0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1])

SINGLE = SphereCase(nx=24, ny=16, nz=16, sphere=(8.0, 8.0, 8.0), radius=3.0, nu=0.01, smagorinsky=0.1)
REFINED = SphereCase(nx=32, ny=16, nz=16, sphere=(10.0, 8.0, 8.0), radius=3.0, nu=0.004, smagorinsky=0.1,
                     refine=((6, 4, 4), (18, 12, 12)))


def test_f64_single_level_matches_double_oracle(orc):
    g = GpuSim(SINGLE, storage="f64")
    o = orc.sim(SINGLE, double=True)
    g.run(60)
    o.run(60)
    f = g.grids[0].fArray  # FP32 view of the FP64 state
    assert np.array_equal(g.shifts(), o.shifts())
    assert rel(f, o.populations()) < 1e-6  # the export rounds to FP32
    m = g.grids[0].macroscopic()
    fo = o.populations()
    rho = fo.sum(0)
    # FP64 state vs FP64 oracle: only double-precision rounding differs
    assert np.max(np.abs(m[0] - rho)) < 1e-12
    assert np.max(np.abs(m[1] - (CX[:, None] * fo).sum(0) / rho)) < 1e-12
    g.close()


def test_f64_two_levels_match_double_oracle(orc):
    g = GpuSim(REFINED, storage="f64")
    o = orc.sim(REFINED, double=True)
    g.run(20)
    o.run(20)
    for lev in range(2):
        fo = o.populations(lev)
        m = g.grids[lev].macroscopic()
        rho = fo.sum(0)
        assert np.max(np.abs(m[0] - rho)) < 1e-12, lev
        for comp, c in ((1, CX), (2, CY), (3, CZ)):
            assert np.max(np.abs(m[comp] - (c[:, None] * fo).sum(0) / rho)) < 1e-12, (lev, comp)
    g.close()


@pytest.mark.parametrize("storage,bound", [("f32", 1e-5), ("f16", 5e-3), ("bf16", 4e-2)])
def test_refined_storage_forms_against_f64(storage, bound):
    ref = GpuSim(REFINED, storage="f64")
    run = GpuSim(REFINED, storage=storage)
    ref.run(40)
    run.run(40)
    err = speed_error(run.grids, ref.grids)
    assert err < bound, (storage, err)
    assert run.grids[0].health() == 0 and run.grids[1].health() == 0
    ref.close()
    run.close()


def test_error_ordering_f32_f16_bf16():
    ref = GpuSim(REFINED, storage="f64")
    ref.run(40)
    errs = {}
    for s in ("f32", "f16", "bf16"):
        run = GpuSim(REFINED, storage=s)
        run.run(40)
        errs[s] = speed_error(run.grids, ref.grids)
        run.close()
    ref.close()
    assert errs["f32"] < errs["f16"] < errs["bf16"], errs


def test_macroscopic_export_matches_population_moments():
    g = GpuSim(SINGLE)
    g.run(10)
    f = g.grids[0].fArray.astype(np.float64)
    m = g.grids[0].macroscopic()
    rho = f.sum(0)
    assert l2rel(m[0], rho) < 1e-12
    assert l2rel(m[1], (CX[:, None] * f).sum(0) / rho) < 1e-10
    assert l2rel(m[3], (CZ[:, None] * f).sum(0) / rho) < 1e-9
    mask = updated_cells(g.grids[0])
    assert mask.sum() == SINGLE.nx * SINGLE.ny * SINGLE.nz  # single level: every cell updated
    g.close()
