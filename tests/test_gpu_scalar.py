"""Scalar transport on the GPU (psl_enable_scalar_transport) against the reference's own
scalar-transport update (include/scalarTransportFunctions.h, compiled for the host), and
the scheme's exact conservation of sum f T."""
import numpy as np
import pytest

from gpu_helpers import GpuSim, rel
from oracle.bindings import SphereCase
from periodicshiftlbm_b200 import (
    GridStruct,
    InfoStruct,
    applyLocalCellUpdate,
    applyStreaming,
    fillEquilibriumFromFunction,
)

pytestmark = pytest.mark.gpu


def test_scalar_transport_run_matches_reference(ref):
    case = SphereCase(nx=28, ny=16, nz=14, sphere=(10.0, 8.0, 7.0), radius=2.5, nu=0.01, wall_mode=1)
    tau_t = 0.8
    g = GpuSim(case)
    grid = g.grids[0]
    grid.enableScalarTransport(tau_t)
    given = np.full((case.nz, case.ny, case.nx), np.nan, dtype=np.float32)
    j = np.arange(case.ny)[None, :]
    given[:, :, 0] = np.where(j < case.ny // 2, 1.0, 0.0)
    grid.setScalarGiven(given.reshape(-1))
    r = ref.sim(case)
    ref.enable_scalar(r, tau_t, inlet=True)
    g.run(30)
    r.run(30)
    assert rel(g.populations(), r.populations()) < 1e-5
    t_gpu, t_ref = grid.TArray, ref.scalar_populations(r)
    assert np.max(np.abs(t_gpu - t_ref)) < 1e-5
    assert t_ref.max() > 0.5  # the inlet concentration has entered
    c = grid.scalar()
    assert np.all(np.isfinite(c)) and c.max() <= 1.0 + 1e-4
    assert grid.health() == 0
    g.close()


def test_scalar_content_is_conserved():
    g = GridStruct(InfoStruct(cellCountX=12, cellCountY=10, cellCountZ=8, nu=0.02))
    fillEquilibriumFromFunction(g, rho=1.0, u=(0.03, -0.02, 0.01))
    g.enableScalarTransport(0.7)
    rng = np.random.default_rng(3)
    g.TArray = np.repeat(rng.uniform(0.0, 1.0, (1, g.cellCount)), 27, axis=0).astype(np.float32)

    def content():
        return float((g.fArray.astype(np.float64) * g.TArray.astype(np.float64)).sum())

    before = content()
    for _ in range(20):
        applyStreaming(g)
        applyLocalCellUpdate(g)
    after = content()
    assert abs(after - before) < 1e-5 * abs(before)
    g.close()
