"""Section-cut export on the GPU against its definition (exportSectionCutPlotGeneral,
plotter/exportSectionCutPlot.h:1-88) evaluated in numpy FP32 with the reference's order of
additions: bit for bit."""
import numpy as np
import pytest

from gpu_helpers import GpuSim
from oracle.bindings import SphereCase
from periodicshiftlbm_b200 import _lib, sectionCut

pytestmark = pytest.mark.gpu

CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1]
CY = [0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1]
CZ = [0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1]


def reference_section(f, solid, plane, cut, rho_nom, cs, res, dt):
    """f [27, z, y, x] float32 -> [V, H, 5] float32 in the reference's arithmetic."""
    if plane == "XY":
        fs, sol = f[:, cut, :, :], solid[cut, :, :]            # [q, y, x]
    elif plane == "ZY":
        fs, sol = f[:, :, :, cut].transpose(0, 2, 1), solid[:, :, cut].T  # [q, y, z]
    else:
        fs, sol = f[:, :, cut, :].transpose(0, 2, 1), solid[:, cut, :].T  # [q, x, z]
    f32 = np.float32
    rho = np.zeros(fs.shape[1:], f32)
    j = [np.zeros(fs.shape[1:], f32) for _ in range(3)]
    for q in range(27):
        rho = rho + fs[q]
        for a, c in enumerate((CX, CY, CZ)):
            if c[q] > 0:
                j[a] = j[a] + fs[q]
            elif c[q] < 0:
                j[a] = j[a] - fs[q]
    u = [ja / rho for ja in j]
    vs = f32(res) / f32(1000.0)
    u = [(ua * vs) / f32(dt) for ua in u]
    p = (rho - f32(1.0)) * (f32(rho_nom) * f32(cs) * f32(cs))
    ux, uy, uz = u
    comps = {"XY": (ux, uy, uz), "ZY": (uz, uy, ux), "ZX": (uz, ux, uy)}[plane]
    return np.stack([p, *comps, sol.astype(f32)], axis=-1)


@pytest.mark.parametrize("plane,cut", [("XY", 7), ("ZY", 11), ("ZX", 6)])
def test_section_cut_bitwise_against_definition(plane, cut):
    c = SphereCase(nx=24, ny=14, nz=12, sphere=(9.0, 7.0, 6.0), radius=3.0, nu=0.01)
    s = GpuSim(c)
    s.run(15)
    g = s.grids[0]
    f = g.fArray.reshape(27, c.nz, c.ny, c.nx)
    solid = (g.markers.reshape(c.nz, c.ny, c.nx) & 7) == _lib.CELL_SOLID
    got = sectionCut(g, plane, cut, rho_nominal_phys=998.0, soundspeed_phys=20.0)
    want = reference_section(f, solid, plane, cut, 998.0, 20.0, g.Info.res, g.Info.dtPhys)
    assert got.shape == want.shape
    assert np.array_equal(got, want)
    assert got[..., 4].sum() > 0  # the sphere shows
    s.close()
