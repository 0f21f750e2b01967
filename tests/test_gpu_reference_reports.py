"""Reports pinned to the reference's own code (compiled into the reference build):

* the section-cut file of exportSectionCutPlotGeneral (include/plotter/exportSectionCutPlot.h:2-89)
  -- the library's export and the reference's, on the same populations, byte for byte, for
  each plane, on the coarse and the fine grid of a refined case;
* getTorque (M35Full/m35Main.cu:176-260, written for PS grids in the reference build with
  its getForcing hook) against psl_forcing_torque on the same state: a forced-velocity
  annulus around a sphere, driven toward solid rotation by the customised update.
"""
import numpy as np
import pytest

from gpu_helpers import GpuSim
from oracle.bindings import SphereCase
from periodicshiftlbm_b200 import _lib, applyLocalCellUpdate, applyStreaming, exportSectionCutPlot, getForcingTorque
from periodicshiftlbm_b200._lib import call
from periodicshiftlbm_b200.grid import MARKER_FORCED_VELOCITY

pytestmark = pytest.mark.gpu

REFINED = SphereCase(nx=32, ny=16, nz=16, sphere=(12.0, 8.0, 8.0), radius=2.5, nu=0.004, smagorinsky=0.1,
                     refine=((6, 4, 4), (18, 12, 12)))


@pytest.mark.parametrize("level,plane,cut", [(0, "XY", 7), (0, "ZY", 11), (0, "ZX", 6), (1, "XY", 9), (1, "ZY", 5),
                                             (1, "ZX", 12)])
def test_section_cut_file_equals_reference_export(ref, tmp_path, level, plane, cut):
    s = GpuSim(REFINED)
    s.run(12)
    g = s.grids[level]
    mine, theirs = str(tmp_path / "mine.bin"), str(tmp_path / "theirs.bin")
    # the reference build's physical constants: rhoNominalPhys = 1.225, soundspeedPhys = 1
    exportSectionCutPlot(g, plane, cut, 7, path=mine, rho_nominal_phys=1.225, soundspeed_phys=1.0)
    r = ref.sim(REFINED)
    r.set_populations(g.fArray, level)  # logical order: independent of the shifts
    r.export_section(level, plane, cut, 7, theirs)
    a, b = open(mine, "rb").read(), open(theirs, "rb").read()
    assert len(a) == len(b)
    assert a == b
    s.close()
    r.close()


def test_forcing_torque_equals_reference_get_torque(ref):
    R0, R1, omega = 4.0, 7.0, 0.004
    case = SphereCase(nx=24, ny=20, nz=16, sphere=(10.0, 10.0, 8.0), radius=2.5, nu=0.01, force_annulus=(R0, R1, omega))
    s = GpuSim(case)
    g = s.grids[0]
    nx, ny, nz = case.nx, case.ny, case.nz
    f32 = np.float32
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    # the reference hooks' FP32 arithmetic: x = i res + ox, annulus test, solid-rotation target
    x = i.astype(f32) * f32(g.Info.res) + f32(g.Info.ox)
    y = j.astype(f32) * f32(g.Info.res) + f32(g.Info.oy)
    dx, dy = x - f32(case.sphere[0]), y - f32(case.sphere[1])
    a2 = dx * dx + dy * dy
    markers = g.markers.reshape(nz, ny, nx)
    forced = (a2 >= f32(R0 * R0)) & (a2 <= f32(R1 * R1)) & ((markers & 7) == _lib.CELL_FLUID)
    markers[forced] = MARKER_FORCED_VELOCITY
    g.markers = markers.reshape(-1)
    given = np.zeros((nz, ny, nx, 4), dtype=f32)
    given[..., 0] = 1.0
    given[..., 1] = -f32(omega) * dy
    given[..., 2] = f32(omega) * dx
    call("psl_set_given_field", g.handle, np.ascontiguousarray(given.reshape(-1, 4)).ctypes.data)
    for _ in range(3):
        applyStreaming(g)
        applyLocalCellUpdate(g)
    torque, force = getForcingTorque(g, k_min=5, rho_nominal_phys=1.225)
    r = ref.sim(case)
    r.set_populations(g.fArray, 0)
    want = r.torque(0)
    assert forced.sum() > 200 and abs(want) > 0
    # the reference sums FP32 terms; the library FP64
    assert torque == pytest.approx(want, rel=2e-5), (torque, want)
    assert np.all(np.isfinite(force))
    s.close()
    r.close()
