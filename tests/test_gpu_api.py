"""Behaviour of the C ABI on the GPU: data movement, markers, periodic fix-up, storage
forms, health flag and error paths."""
import ctypes

import numpy as np
import pytest

from gpu_helpers import GpuSim, rel
from oracle.bindings import SphereCase
from periodicshiftlbm_b200 import (
    GridStruct,
    InfoStruct,
    _lib,
    applyBCPeriodicX,
    applyBCPeriodicY,
    applyCoarseFineGridCommunication,
    applyLocalCellUpdate,
    applyStreaming,
    fillEquilibriumFromFunction,
)
from periodicshiftlbm_b200.cases import config1, make_sphere_grids

pytestmark = pytest.mark.gpu


def test_populations_roundtrip_f32_bit_exact():
    g = GridStruct(InfoStruct(cellCountX=10, cellCountY=7, cellCountZ=5, nu=0.01))
    rng = np.random.default_rng(1)
    f = rng.uniform(0.0, 0.3, (27, g.cellCount)).astype(np.float32)
    for _ in range(3):
        applyStreaming(g)  # non-trivial shifts
    g.fArray = f
    assert np.array_equal(g.fArray, f)


@pytest.mark.parametrize("storage,tol", [("f16", 1e-3), ("bf16", 8e-3)])
def test_shifted_storage_roundtrip(storage, tol):
    g = GridStruct(InfoStruct(cellCountX=10, cellCountY=7, cellCountZ=5, nu=0.01), storage=storage)
    fillEquilibriumFromFunction(g, rho=1.0, u=(0.05, -0.02, 0.01))
    f = g.fArray
    ref = GridStruct(InfoStruct(cellCountX=10, cellCountY=7, cellCountZ=5, nu=0.01))
    fillEquilibriumFromFunction(ref, rho=1.0, u=(0.05, -0.02, 0.01))
    fr = ref.fArray
    # |f - w| is stored, so the absolute error is a fraction of |f - w|, not of f
    w = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)[:, None]
    assert np.max(np.abs(f - fr) / np.maximum(np.abs(fr - w), 1e-4)) < tol


def test_markers_match_sphere_hooks():
    cfg = config1()
    grids, _ = make_sphere_grids(cfg)
    m = grids[0].markers.reshape(cfg.nz, cfg.ny, cfg.nx)
    k, j, i = np.meshgrid(np.arange(cfg.nz), np.arange(cfg.ny), np.arange(cfg.nx), indexing="ij")
    r2 = (i - 32.0) ** 2 + (j - 32.0) ** 2 + (k - 32.0) ** 2
    kind = m & 7
    assert np.all(kind[r2 <= 64] == _lib.CELL_SOLID)
    assert np.sum(kind == _lib.CELL_SOLID) == np.sum(r2 <= 64)
    assert np.all(kind[:, :, 0] == _lib.CELL_GIVEN_U)
    assert np.all(kind[:, :, -1] == _lib.CELL_GIVEN_RHO)
    wall = (j == 0) | (j == cfg.ny - 1) | (k == 0) | (k == cfg.nz - 1)
    inner_x = (i > 0) & (i < cfg.nx - 1)
    assert np.all(kind[wall & inner_x] == _lib.CELL_MIRROR)
    # outer normal of the y=0, z=0 edge: (0,-1,-1) -> index 9*1 + 3*0 + 0 = 9
    assert m[0, 0, 5] >> 3 == 9
    assert np.all(kind[~wall & inner_x & (r2 > 64)] == _lib.CELL_FLUID)


def test_periodic_fixup_matches_reference(ref):
    """applyBCPeriodicX/Y copy populations between the two faces (copies only: exact)."""
    c = SphereCase(nx=10, ny=8, nz=6, sphere=(100.0, 100.0, 100.0), radius=1.0, nu=0.01)
    r = ref.sim(c)
    g = GpuSim(c)
    rng = np.random.default_rng(3)
    f = rng.uniform(0.0, 0.3, (27, 480)).astype(np.float32)
    r.set_populations(f)
    g.grids[0].fArray = f
    for axis in (0, 1):
        ref.lib.ref_sim_streaming(r.h, 0)
        applyStreaming(g.grids[0])
        if axis == 0:
            ref.lib.ref_sim_periodic_x(r.h, 0)
            applyBCPeriodicX(g.grids[0])
        else:
            ref.lib.ref_sim_periodic_y(r.h, 0)
            applyBCPeriodicY(g.grids[0])
        assert np.array_equal(g.populations(), r.populations()), axis
    g.close()


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_reduced_storage_run_tracks_fp32(storage):
    c = SphereCase(nx=24, ny=16, nz=16, sphere=(8.0, 8.0, 8.0), radius=3.0, nu=0.01)
    a = GpuSim(c)
    b = GpuSim(c, storage=storage)
    a.run(100)
    b.run(100)
    fa, fb = a.populations(), b.populations()
    ua = (fa * np.array(_cx())[:, None]).sum(0) / fa.sum(0)
    ub = (fb * np.array(_cx())[:, None]).sum(0) / fb.sum(0)
    err = np.linalg.norm(ua - ub) / np.linalg.norm(ua)
    assert err < (2e-3 if storage == "f16" else 2e-2), err
    a.close()
    b.close()


def _cx():
    return [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1]


def test_health_flag_reports_non_finite_state():
    """Failure detection: a non-finite population planted in the host input makes the
    update kernel raise the health bit; the context stays usable."""
    g = GridStruct(InfoStruct(cellCountX=8, cellCountY=8, cellCountZ=8, nu=0.01))
    fillEquilibriumFromFunction(g, rho=1.0, u=(0.01, 0.0, 0.0))
    assert g.health() == 0
    applyStreaming(g)
    applyLocalCellUpdate(g)
    assert g.health() == 0
    f = g.fArray
    f[3, 100] = np.nan
    g.fArray = f
    applyStreaming(g)
    applyLocalCellUpdate(g)
    assert g.health() & 1
    assert g.health() == 0  # read-and-clear
    g.fArray = np.nan_to_num(f, nan=1.0 / 54)
    applyStreaming(g)
    applyLocalCellUpdate(g)
    assert g.health() == 0


def test_coarse_fine_rejects_mismatched_grids():
    c = GridStruct(InfoStruct(cellCountX=16, cellCountY=16, cellCountZ=16, nu=0.01, iSubgridStart=4, jSubgridStart=4,
                              kSubgridStart=4, iSubgridEnd=10, jSubgridEnd=10, kSubgridEnd=10))
    f = GridStruct(InfoStruct(gridID=1, res=0.5, cellCountX=10, cellCountY=12, cellCountZ=12, nu=0.02))
    with pytest.raises(_lib.PslError):
        applyCoarseFineGridCommunication(c, f)


def test_set_shifts_validates_range():
    g = GridStruct(InfoStruct(cellCountX=4, cellCountY=4, cellCountZ=4, nu=0.01))
    with pytest.raises(_lib.PslError):
        g.shifter = np.full(27, 64, dtype=np.int32)


def test_plain_kernel_on_grid_not_multiple_of_tile(orc):
    """N % 4 != 0 takes the one-thread-per-cell kernel; it still matches the oracle."""
    c = SphereCase(nx=13, ny=9, nz=7, sphere=(5.0, 4.0, 3.0), radius=1.5, nu=0.02)
    g = GpuSim(c)
    o = orc.sim(c)
    g.run(50)
    o.run(50)
    assert rel(g.populations(), o.populations()) < 1e-5
    g.close()



def test_async_sphere_force_matches_synchronous():
    """psl_sphere_force_async into pinned host memory and into device memory, several steps
    queued before one synchronisation, equals psl_sphere_force step by step."""
    import torch

    from periodicshiftlbm_b200 import getSphereForce, getSphereForceAsync, updateGrid

    cfg = config1(nx=48, ny=24, nz=24, sphere=(12.0, 12.0, 12.0), radius=4.0)
    ga, case = make_sphere_grids(cfg)
    gb, _ = make_sphere_grids(cfg)
    steps = 6
    host = torch.zeros((steps, 3), dtype=torch.float64).pin_memory()
    dev = torch.zeros((steps, 3), dtype=torch.float64, device="cuda")
    want = []
    for s in range(steps):
        updateGrid(ga, 0)
        want.append(getSphereForce(ga[0], case))
        updateGrid(gb, 0)
        getSphereForceAsync(gb[0], case, host.data_ptr() + 24 * s)
        getSphereForceAsync(gb[0], case, dev.data_ptr() + 24 * s)
    gb[0].synchronize()
    assert np.array_equal(host.numpy(), np.array(want))
    assert np.array_equal(dev.cpu().numpy(), np.array(want))
    assert np.all(np.array(want)[:, 0] != 0.0)
    for g in ga + gb:
        g.close()
