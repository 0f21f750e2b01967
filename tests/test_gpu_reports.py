"""FP64 report reductions on the GPU: torque/force of the momentum exchange and the plane
flow report, against numpy on the exported populations and markers."""
import numpy as np
import pytest

from gpu_helpers import GpuSim
from oracle.bindings import SphereCase
from periodicshiftlbm_b200 import getFlowReport, getSphereForce, getTorque, _lib

pytestmark = pytest.mark.gpu

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1])
CZ = np.array([0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1])


def moments(g):
    info = g.Info
    f = g.fArray.astype(np.float64).reshape(27, info.cellCountZ, info.cellCountY, info.cellCountX)
    rho = f.sum(0)
    j = np.stack([np.tensordot(c, f, 1) for c in (CX, CY, CZ)])
    solid = (g.markers.reshape(rho.shape) & 7) == _lib.CELL_SOLID
    return rho, j, solid


def test_torque_and_force_match_numpy():
    c = SphereCase(nx=32, ny=20, nz=18, sphere=(10.0, 9.5, 8.5), radius=4.0, nu=0.01)
    s = GpuSim(c)
    s.run(30)
    g = s.grids[0]
    rho, j, solid = moments(g)
    lo, hi, pt = (4, 3, 2), (18, 17, 15), (10.0, 9.5, 8.5)
    box = np.zeros_like(solid)
    box[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = True
    sel = solid & box
    k, jj, i = np.nonzero(sel)
    F = 2.0 * j[:, sel]
    r = np.stack([i - pt[0], jj - pt[1], k - pt[2]]).astype(np.float64)
    want_t = np.cross(r.T, F.T).sum(0)
    t, f = getTorque(g, lo, hi, pt)
    assert np.allclose(f, F.sum(1), rtol=1e-12, atol=1e-15)
    assert np.allclose(t, want_t, rtol=1e-10, atol=1e-13)
    # the sphere's own box: the force is the drag reduction's
    sf = getSphereForce(g, s.sc)
    t2, f2 = getTorque(g, (0, 0, 0), (32, 20, 18), pt)
    assert np.allclose(f2, sf, rtol=1e-12, atol=1e-14)
    s.close()


@pytest.mark.parametrize("plane,cut", [("XY", 9), ("ZY", 12), ("ZX", 7)])
def test_flow_report_single_level_matches_numpy(plane, cut):
    c = SphereCase(nx=28, ny=18, nz=16, sphere=(12.0, 9.0, 8.0), radius=4.0, nu=0.01)
    s = GpuSim(c)
    s.run(20)
    g = s.grids[0]
    rho, j, solid = moments(g)
    u = j / rho
    if plane == "XY":
        sl = (cut, slice(None), slice(None))
    elif plane == "ZY":
        sl = (slice(None), slice(None), cut)
    else:
        sl = (slice(None), cut, slice(None))
    keep = ~solid[sl]
    rep = getFlowReport([g], plane, cut, (-1, -1, -1, 100, 100, 100))
    assert rep["area"] == pytest.approx(keep.sum())
    for comp, name in enumerate(("ux", "uy", "uz")):
        assert rep[name] == pytest.approx(u[comp][sl][keep].mean(), rel=1e-6, abs=1e-9)
    assert rep["rho"] == pytest.approx((rho[sl][keep] - 1.0).mean() + 1.0, rel=1e-7)
    s.close()


def test_flow_report_two_levels_uses_the_fine_grid_inside_the_block():
    c = SphereCase(nx=32, ny=16, nz=16, sphere=(10.0, 8.0, 8.0), radius=3.0, nu=0.004, smagorinsky=0.1,
                   refine=((6, 4, 4), (18, 12, 12)))
    s = GpuSim(c)
    s.run(10)
    fine = s.grids[1]
    rho, j, solid = moments(fine)
    cut = 9  # finest-grid z index
    keep = ~solid[cut]
    rep = getFlowReport(s.grids, "XY", cut, (-100, -100, -100, 100, 100, 100))
    assert rep["area"] == pytest.approx(keep.sum() * 0.25)
    assert rep["ux"] == pytest.approx((j[0] / rho)[cut][keep].mean(), rel=1e-6)
    s.close()


@pytest.mark.parametrize("plane,cut,bounds", [("XY", 9, (-1, -1, -1, 100, 100, 100)),
                                              ("ZY", 12, (-1, -1, -1, 100, 100, 100)),
                                              ("ZX", 7, (-1, -1, -1, 100, 100, 100)),
                                              ("XY", 8, (6.5, 3.2, -1, 21.7, 14.1, 100)),
                                              ("ZY", 15, (-1, 2.5, 4.0, 100, 15.5, 12.2))])
def test_flow_report_matches_the_reference_function(ref, plane, cut, bounds):
    """psl_get_flow_report of one level against the reference's own getFlowReportGeneral
    (flowReportFunctions.h:2-251) compiled for the host, run on a one-level DIAD grid that
    holds the same state (the PS grid's populations after 20 steps); the reference sums in
    FP32, this library in FP64."""
    c = SphereCase(nx=28, ny=18, nz=16, sphere=(12.0, 9.0, 8.0), radius=4.0, nu=0.01)
    s = GpuSim(c)
    s.run(20)
    g = s.grids[0]
    r = ref.sim(c)
    r.set_populations(g.fArray, 0)
    want = r.flow_report(0, plane, cut, bounds)
    got = getFlowReport([g], plane, cut, bounds)
    assert got["area"] == want["area"] and want["area"] > 0
    for name in ("ux", "uy", "uz", "rho"):
        assert got[name] == pytest.approx(want[name], rel=2e-5, abs=1e-7), (name, got[name], want[name])
    r.close()
    s.close()
