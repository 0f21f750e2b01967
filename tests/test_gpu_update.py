"""The update kernel on arbitrary shifts and the per-cell Smagorinsky hook.

* Grids and shifts that exercise the shifted addressing -- one 128-cell block, several
  blocks with a partial last one, shifts whose wrap point falls inside a block or between
  the two cells of a pair, an odd cell count, arbitrary shifts -- for every storage form, with and without a per-cell C_s
  field, with skipped and solid cells among the fluid ones: every cell against the
  oracle's collision (FP64), skipped cells unchanged and solid cells bounced back bit for
  bit.
* A refined LES sphere run whose coarse grid has a per-cell C_s (a sponge ahead of the
  outlet, getSmagorinskyConstant per cell) against the reference's own update run live.
"""
import numpy as np
import pytest

from gpu_helpers import GpuSim, rel
from oracle.bindings import SphereCase
from periodicshiftlbm_b200 import GridStruct, InfoStruct, applyLocalCellUpdate
from periodicshiftlbm_b200 import _lib
from periodicshiftlbm_b200.grid import setSmagorinskyConstant

pytestmark = pytest.mark.gpu

W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
OPP = np.array([0] + [q + 1 if q % 2 else q - 1 for q in range(1, 27)])
# |f_out - want| bound per storage: FP32 arithmetic, or the 16-bit rounding of g = f - w
# (|g| < 0.03 here: FP16 half-ulp 7.6e-6, BF16 6.1e-5)
TOL = {"f32": ("rel", 2e-6), "f16": ("abs", 2e-5), "bf16": ("abs", 2.5e-4)}


def _start(orc, n, rng):
    f = np.empty((27, n))
    for c in range(n):
        rho = 1.0 + rng.uniform(-0.01, 0.01)
        f[:, c] = orc.feq(rho, *rng.uniform(-0.06, 0.06, 3), dtype=np.float64)
    return (f * (1.0 + rng.uniform(-2e-3, 2e-3, f.shape))).astype(np.float32)


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("dims", [(12, 4, 2), (20, 3, 8), (16, 8, 8), (40, 12, 12), (7, 5, 3)])
@pytest.mark.parametrize("field", [False, True])
def test_update_matches_oracle_for_any_shift(orc, storage, dims, field):
    nx, ny, nz = dims
    n = nx * ny * nz
    nu, cs = 0.004, 0.12
    rng = np.random.default_rng(n + 7 * len(storage) + field)
    g = GridStruct(InfoStruct(cellCountX=nx, cellCountY=ny, cellCountZ=nz, nu=nu), storage=storage)
    shifts = rng.integers(0, n, 27)
    shifts[1:6] = n - 1 - np.arange(5)  # wrap points inside the first block
    shifts[0] = 0
    g.shifter = shifts.astype(np.int32)
    assert np.array_equal(g.shifter, shifts)
    kinds = np.full(n, _lib.CELL_FLUID, dtype=np.uint8)
    kinds[rng.random(n) < 0.08] = _lib.CELL_SKIP
    kinds[rng.random(n) < 0.08] = _lib.CELL_SOLID
    g.markers = kinds
    cs_cell = rng.uniform(0.0, 0.25, n).astype(np.float32) if field else np.full(n, cs, np.float32)
    setSmagorinskyConstant(g, cs_cell if field else cs)
    g.fArray = _start(orc, n, rng)
    f_in = g.fArray  # as stored (rounded for the 16-bit forms)
    applyLocalCellUpdate(g)
    out = g.fArray
    assert g.health() == 0
    skip = kinds == _lib.CELL_SKIP
    solid = kinds == _lib.CELL_SOLID
    assert np.array_equal(out[:, skip], f_in[:, skip])
    assert np.array_equal(out[:, solid], f_in[OPP][:, solid])
    mode, tol = TOL[storage]
    for c in np.flatnonzero(kinds == _lib.CELL_FLUID)[:: max(1, n // 300)]:
        want = orc.collision(f_in[:, c].astype(np.float64), nu, float(cs_cell[c]), dtype=np.float64)
        err = np.abs(out[:, c] - want)
        if mode == "rel":
            err = err / np.abs(want)
        assert err.max() < tol, (c, err.max())
    g.close()


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_16bit_health_flag(storage):
    g = GridStruct(InfoStruct(cellCountX=16, cellCountY=8, cellCountZ=8, nu=0.01), storage=storage)
    f = np.tile(W.astype(np.float32)[:, None], (1, g.cellCount))
    f[5, 77] = np.nan
    g.fArray = f
    applyLocalCellUpdate(g)
    assert g.health() & 1
    assert g.health() == 0
    g.close()


def test_per_cell_smagorinsky_sphere_matches_reference(ref):
    case = SphereCase(nx=32, ny=16, nz=16, sphere=(12.0, 8.0, 8.0), radius=2.5, nu=0.002, smagorinsky=0.15,
                      cs_mode=1, refine=((6, 4, 4), (18, 12, 12)))
    g = GpuSim(case)
    r = ref.sim(case)
    g.run(60)
    r.run(60)
    for lev in range(2):
        assert np.array_equal(g.shifts(lev), r.shifts(lev))
        assert rel(g.populations(lev), r.populations(lev)) < 1e-5, lev
    g.close()
    r.close()

