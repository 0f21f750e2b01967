"""Host-side mirror of the reference's per-step update API, over the C ABI.

Names, argument meaning and call order follow the reference's free functions
(include/applyStreaming.h, include/applyLocalCellUpdate.h, include/fillEquilibrium.h,
include/gridRefinementFunctions.h, include/boundaryConditions/periodicXY.h) and the case
driver's updateGrid recursion (flowAroundSphere/flowAroundSphereMainSingle.cu:158-167), so
a driver reads like the reference's:

    grids = [GridStruct(info0), GridStruct(info1)]
    for g in grids:
        setSphereCase(g, case)                 # getMarkers / getGiven... hooks
        fillEquilibriumFromFunction(g, case)   # getInitialRhoUxUyUz hook
    for it in range(steps):
        updateGrid(grids, 0)
        drag = getSphereDrag(grids[-1], case)

Every call goes to the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import PslInfo, PslSphereCase, call


@dataclass
class InfoStruct:
    """Mirrors InfoStruct (include/types.h:73-75)."""

    gridID: int = 0
    res: float = 1.0
    cellCountX: int = 0
    cellCountY: int = 0
    cellCountZ: int = 0
    ox: float = 0.0
    oy: float = 0.0
    oz: float = 0.0
    nu: float = 1.0
    dtPhys: float = 1.0
    iSubgridStart: int = 0
    jSubgridStart: int = 0
    kSubgridStart: int = 0
    iSubgridEnd: int = 0
    jSubgridEnd: int = 0
    kSubgridEnd: int = 0

    @property
    def cellCount(self) -> int:
        return self.cellCountX * self.cellCountY * self.cellCountZ

    def to_c(self) -> PslInfo:
        c = PslInfo()
        c.grid_id = int(self.gridID)
        c.res = self.res
        c.cell_count_x, c.cell_count_y, c.cell_count_z = self.cellCountX, self.cellCountY, self.cellCountZ
        c.ox, c.oy, c.oz = self.ox, self.oy, self.oz
        c.nu = self.nu
        c.dt_phys = self.dtPhys
        c.i_subgrid_start, c.j_subgrid_start, c.k_subgrid_start = (
            self.iSubgridStart, self.jSubgridStart, self.kSubgridStart)
        c.i_subgrid_end, c.j_subgrid_end, c.k_subgrid_end = self.iSubgridEnd, self.jSubgridEnd, self.kSubgridEnd
        return c

    def finer(self) -> "InfoStruct":
        """Metadata of the 2:1 refined grid over this grid's subgrid block
        (flowAroundSphereMainSingle.cu:185-215): half the cell size and time step, twice
        the lattice viscosity, origin half a fine cell inside the block."""
        f = InfoStruct()
        f.gridID = self.gridID + 1
        f.res = np.float32(self.res * np.float32(0.5)).item()
        f.dtPhys = np.float32(self.dtPhys * np.float32(0.5)).item()
        f.nu = np.float32(self.nu * np.float32(2.0)).item()
        f32 = np.float32
        f.ox = float(f32(f32(self.ox) + f32(self.iSubgridStart) * f32(self.res)) - f32(f.res) * f32(0.5))
        f.oy = float(f32(f32(self.oy) + f32(self.jSubgridStart) * f32(self.res)) - f32(f.res) * f32(0.5))
        f.oz = float(f32(f32(self.oz) + f32(self.kSubgridStart) * f32(self.res)) - f32(f.res) * f32(0.5))
        f.cellCountX = (self.iSubgridEnd - self.iSubgridStart) * 2
        f.cellCountY = (self.jSubgridEnd - self.jSubgridStart) * 2
        f.cellCountZ = (self.kSubgridEnd - self.kSubgridStart) * 2
        return f


@dataclass
class SphereCase:
    """The flow-past-sphere hooks (flowAroundSphere/flowAroundSphereMainSingle.cu:41-92)."""

    sphere: tuple = (32.0, 32.0, 32.0)  # physical centre
    radius: float = 8.0
    u_in: float = 0.05
    rho_given: float = 1.0
    wall_mode: int = 0       # 0 free-slip y/z walls, 1 velocity walls
    smagorinsky: float = 0.0
    seed: int = 1234
    noise: float = 1e-4

    def to_c(self) -> PslSphereCase:
        c = PslSphereCase()
        c.sphere_x, c.sphere_y, c.sphere_z = self.sphere
        c.sphere_r = self.radius
        c.u_in = self.u_in
        c.rho_given = self.rho_given
        c.wall_mode = self.wall_mode
        c.smagorinsky = self.smagorinsky
        c.seed = self.seed
        c.noise_amp = self.noise
        return c


class GridStruct:
    """One PS grid on the GPU (GridStruct, include/types.h:77): metadata, the [27][N]
    population array and the 27 periodic shifts.  Owns its device memory."""

    def __init__(self, Info: InfoStruct, storage: str = "f32", one_mapping: bool = False):
        """``one_mapping``: keep the population rows in one plain allocation even where they
        could be mapped twice (psl.h, psl_grid_create_ex); the results are the same bits."""
        self.Info = Info
        self.storage = storage
        self._h = ctypes.c_void_p()
        call("psl_grid_create_ex", ctypes.byref(Info.to_c()), _lib.STORAGE[storage],
             ctypes.c_uint(1 if one_mapping else 0), ctypes.byref(self._h))

    @property
    def rows_mapped_twice(self) -> bool:
        """Whether the population rows are mapped twice (the update then reads them without
        the periodic wrap)."""
        twice = ctypes.c_int()
        call("psl_grid_get_layout", self._h, ctypes.byref(twice), None)
        return bool(twice.value)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h and self._h.value:
            call("psl_grid_destroy", self._h)  # refuses (raises) while the grid is in a batch
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def cellCount(self) -> int:
        return self.Info.cellCount

    # fArray / shifter accessors (logical cell order)
    @property
    def fArray(self) -> np.ndarray:
        out = np.empty((27, self.cellCount), dtype=np.float32)
        call("psl_get_populations", self._h, out.ctypes.data)
        return out

    @fArray.setter
    def fArray(self, f: np.ndarray):
        f = np.ascontiguousarray(f, dtype=np.float32).reshape(27, self.cellCount)
        call("psl_set_populations", self._h, f.ctypes.data)

    def read_populations(self, out: np.ndarray) -> np.ndarray:
        """fArray into a caller-provided float32 [27][N] buffer (e.g. pinned host memory)."""
        assert out.dtype == np.float32 and out.size == 27 * self.cellCount and out.flags.c_contiguous
        call("psl_get_populations", self._h, out.ctypes.data)
        return out

    def write_populations(self, src: np.ndarray):
        """Set fArray from a caller-provided float32 [27][N] buffer."""
        assert src.dtype == np.float32 and src.size == 27 * self.cellCount and src.flags.c_contiguous
        call("psl_set_populations", self._h, src.ctypes.data)

    def macroscopic(self) -> np.ndarray:
        """(rho, ux, uy, uz) of every cell, [4][N] float64 in logical order, summed in FP64
        from the stored populations (getRhoUxUyUz, cellFunctions.h:135-155)."""
        out = np.empty((4, self.cellCount), dtype=np.float64)
        call("psl_get_macroscopic", self._h, out.ctypes.data)
        return out

    # ---- scalar transport (scalarTransportFunctions.h) ----
    def enableScalarTransport(self, tauT: float):
        """27 scalar populations T_q streamed with f and collided after it (relaxation tauT)."""
        call("psl_enable_scalar_transport", self._h, ctypes.c_float(tauT))

    def setScalarGiven(self, givenT: np.ndarray | None):
        """Per-cell prescribed concentration (NaN: none), or None to remove it."""
        if givenT is None:
            call("psl_set_scalar_given_field", self._h, None)
        else:
            a = np.ascontiguousarray(givenT, dtype=np.float32).reshape(self.cellCount)
            call("psl_set_scalar_given_field", self._h, a.ctypes.data)

    @property
    def TArray(self) -> np.ndarray:
        out = np.empty((27, self.cellCount), dtype=np.float32)
        call("psl_get_scalar_populations", self._h, out.ctypes.data)
        return out

    @TArray.setter
    def TArray(self, t: np.ndarray):
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(27, self.cellCount)
        call("psl_set_scalar_populations", self._h, t.ctypes.data)

    def scalar(self) -> np.ndarray:
        """Concentration of every cell, sum f T / rho (FP64)."""
        out = np.empty(self.cellCount, dtype=np.float64)
        call("psl_get_scalar", self._h, out.ctypes.data)
        return out

    @property
    def shifter(self) -> np.ndarray:
        out = np.zeros(27, dtype=np.int32)
        call("psl_get_shifts", self._h, out.ctypes.data)
        return out

    @shifter.setter
    def shifter(self, s):
        s = np.ascontiguousarray(s, dtype=np.int32)
        call("psl_set_shifts", self._h, s.ctypes.data)

    @property
    def markers(self) -> np.ndarray:
        out = np.empty(self.cellCount, dtype=np.uint8)
        call("psl_get_markers", self._h, out.ctypes.data)
        return out

    @markers.setter
    def markers(self, m):
        m = np.ascontiguousarray(m, dtype=np.uint8)
        call("psl_set_markers", self._h, m.ctypes.data)

    def set_stream(self, stream_ptr: int):
        call("psl_grid_set_stream", self._h, ctypes.c_void_p(stream_ptr))

    def synchronize(self):
        call("psl_synchronize", self._h)

    def health(self) -> int:
        v = ctypes.c_uint(0)
        call("psl_check_health", self._h, ctypes.byref(v))
        return v.value


# ---- hooks ----------------------------------------------------------------------------
def setSphereCase(grid: GridStruct, case: SphereCase):
    """getMarkers / getGivenRhoUxUyUz / getSmagorinskyConstant of the sphere case."""
    call("psl_apply_sphere_case", grid.handle, ctypes.byref(case.to_c()))


def setGivenRhoUxUyUz(grid: GridStruct, rho, ux, uy, uz):
    call("psl_set_given", grid.handle, rho, ux, uy, uz)


def setBodyForce(grid: GridStruct, gx: float, gy: float, gz: float):
    """Uniform body force (lattice units) of the customised update (psl_set_body_force)."""
    call("psl_set_body_force", grid.handle, gx, gy, gz)


MARKER_MOVING_WALL = _lib.CELL_SOLID | (1 << 3)
MARKER_FORCED_VELOCITY = _lib.CELL_FLUID | (1 << 3)


def setSmagorinskyConstant(grid: GridStruct, cs):
    """getSmagorinskyConstant: a number (uniform), a per-cell array of N constants in cell
    order (i fastest), or the hook itself, a function (i, j, k, Info) -> C_s evaluated for
    every cell as the reference does (include/applyLocalCellUpdate.h:68).  None removes a
    per-cell field."""
    if cs is None:
        call("psl_set_smagorinsky_field", grid.handle, None)
        return
    if callable(cs):
        info = grid.Info
        k, j, i = np.meshgrid(np.arange(info.cellCountZ), np.arange(info.cellCountY), np.arange(info.cellCountX),
                              indexing="ij")
        vals = np.array([cs(int(a), int(b), int(c), info) for a, b, c in zip(i.ravel(), j.ravel(), k.ravel())],
                        dtype=np.float32)
        cs = vals
    if np.ndim(cs) == 0:
        call("psl_set_smagorinsky_field", grid.handle, None)
        call("psl_set_smagorinsky", grid.handle, float(cs))
        return
    a = np.ascontiguousarray(cs, dtype=np.float32).reshape(grid.cellCount)
    call("psl_set_smagorinsky_field", grid.handle, a.ctypes.data)


# ---- per-step update --------------------------------------------------------------------
def fillEquilibriumFromFunction(grid: GridStruct, case: SphereCase | None = None, rho=1.0, u=(0.0, 0.0, 0.0)):
    """fillEquilibrium.h:1-22: feq of the start hook (the sphere case's noisy inflow), or
    of a uniform (rho, u) when no case is given."""
    if case is not None:
        call("psl_fill_equilibrium_sphere", grid.handle, ctypes.byref(case.to_c()))
    else:
        call("psl_fill_equilibrium_uniform", grid.handle, rho, *u)


def applyStreaming(grid: GridStruct):
    """applyStreaming.h:11-31 (updates the 27 shifts)."""
    call("psl_apply_streaming", grid.handle)


def applyLocalCellUpdate(grid: GridStruct):
    """applyLocalCellUpdate.h:1-74 (one fused kernel)."""
    call("psl_apply_local_cell_update", grid.handle)


def applyBCPeriodicX(grid: GridStruct):
    call("psl_apply_bc_periodic_x", grid.handle)


def applyBCPeriodicY(grid: GridStruct):
    call("psl_apply_bc_periodic_y", grid.handle)


def applyCoarseFineGridCommunication(coarse: GridStruct, fine: GridStruct):
    """gridRefinementFunctions.h:433-526 (one kernel)."""
    call("psl_apply_coarse_fine_grid_communication", coarse.handle, fine.handle)


def fillCoarseGridFromFine(coarse: GridStruct, fine: GridStruct):
    """gridRefinementFunctions.h:528-535: the coarse cells inside the refinement block take
    the rescaled average of their fine children (the reference calls it before exporting the
    coarse level)."""
    call("psl_fill_coarse_grid_from_fine", coarse.handle, fine.handle)


def updateGrid(grids, level: int = 0):
    """The driver's updateGrid recursion (flowAroundSphereMainSingle.cu:158-167), run in
    the library so one call issues a whole coarse step."""
    arr = (ctypes.c_void_p * len(grids))(*[g.handle.value for g in grids])
    call("psl_update_grid", arr, len(grids), level)


# ---- reductions --------------------------------------------------------------------------
def getSphereForce(grid: GridStruct, case: SphereCase) -> np.ndarray:
    """Momentum-exchange force on the sphere's solid cells, FP64, lattice units of `grid`."""
    out = np.zeros(3, dtype=np.float64)
    call("psl_sphere_force", grid.handle, ctypes.byref(case.to_c()), out.ctypes.data)
    return out


def getSphereForceAsync(grid: GridStruct, case: SphereCase, out_ptr: int):
    """Enqueue the sphere force on the grid's stream into 3 doubles at `out_ptr` (device
    memory or pinned host memory, e.g. a pinned torch tensor's data_ptr()); valid after
    ``grid.synchronize()``.  No host wait."""
    call("psl_sphere_force_async", grid.handle, ctypes.byref(case.to_c()), ctypes.c_void_p(out_ptr))


def getSphereDrag(grid: GridStruct, case: SphereCase) -> float:
    """getSphereDrag (flowAroundSphereMainSingle.cu:99-156), in lattice units of `grid`
    (before convertToPhysicalForce)."""
    return float(getSphereForce(grid, case)[0])


def getTorque(grid: GridStruct, lo, hi, point) -> tuple:
    """(torque[3], force[3]) of the momentum exchange on the solid cells of the box
    [lo, hi) about `point` (psl_torque; getTorque, M35Full/m35Main.cu:176-260)."""
    lo = np.ascontiguousarray(lo, dtype=np.int32)
    hi = np.ascontiguousarray(hi, dtype=np.int32)
    pt = np.ascontiguousarray(point, dtype=np.float32)
    t = np.zeros(3)
    f = np.zeros(3)
    call("psl_torque", grid.handle, lo.ctypes.data, hi.ctypes.data, pt.ctypes.data, t.ctypes.data, f.ctypes.data)
    return t, f


def getForcingTorque(grid: GridStruct, k_min: int = 5, rho_nominal_phys: float = 1.225) -> tuple:
    """getTorque (M35Full/m35Main.cu:176-260) on a PS grid (psl_forcing_torque): the torque
    -g_x y + g_y x of the forced-velocity cells' forcing in N m, and the summed forcing."""
    t = np.zeros(1)
    f = np.zeros(3)
    call("psl_forcing_torque", grid.handle, int(k_min), float(rho_nominal_phys), t.ctypes.data, f.ctypes.data)
    return float(t[0]), f


PLANES = {"XY": 0, "ZY": 1, "ZX": 2}


def getFlowReport(grids, plane: str, cut_index: int, bounds) -> dict:
    """getFlowReportGeneral (flowReportFunctions.h:2-251) over the grid hierarchy `grids`
    (coarsest first): mean ux, uy, uz, rho and the area of the section at finest index
    `cut_index`, bounds = (xmin, ymin, zmin, xmax, ymax, zmax) physical."""
    arr = (ctypes.c_void_p * len(grids))(*[g.handle.value for g in grids])
    b = np.ascontiguousarray(bounds, dtype=np.float32)
    r = _lib.PslFlowReport()
    call("psl_get_flow_report", arr, len(grids), PLANES[plane], int(cut_index), b.ctypes.data, ctypes.byref(r))
    return {"ux": r.ux, "uy": r.uy, "uz": r.uz, "rho": r.rho, "area": r.area}


def sectionCut(grid: GridStruct, plane: str, cut_index: int, rho_nominal_phys: float = 1000.0,
               soundspeed_phys: float = 1.0) -> np.ndarray:
    """The section of exportSectionCutPlotGeneral (plotter/exportSectionCutPlot.h:1-88) as a
    [vertical, horizontal, 5] float32 array: p, u_horizontal, u_vertical, u_normal, solid."""
    v, h = ctypes.c_int(), ctypes.c_int()
    call("psl_export_section_cut", grid.handle, PLANES[plane], int(cut_index), rho_nominal_phys, soundspeed_phys,
         None, 0, ctypes.byref(v), ctypes.byref(h))
    out = np.empty((v.value, h.value, 5), dtype=np.float32)
    call("psl_export_section_cut", grid.handle, PLANES[plane], int(cut_index), rho_nominal_phys, soundspeed_phys,
         out.ctypes.data, out.size, ctypes.byref(v), ctypes.byref(h))
    return out


def write_section_cut(path: str, plot_number: int, section: np.ndarray):
    """The file the reference's plotters read (exportSectionCutPlot.h:64-88, plotter.py):
    int32 {plot number, vertical, horizontal, 5}, then the float32 records row by row."""
    section = np.ascontiguousarray(section, dtype=np.float32)
    with open(path, "wb") as fh:
        np.array([plot_number, section.shape[0], section.shape[1], section.shape[2]], dtype=np.int32).tofile(fh)
        section.tofile(fh)


def exportSectionCutPlot(grid: GridStruct, plane: str, cut_index: int, plot_number: int,
                         path: str = "/dev/shm/sim_data.bin", rho_nominal_phys: float = 1000.0,
                         soundspeed_phys: float = 1.0) -> np.ndarray:
    """exportSectionCutPlotXY/ZY/ZX: the section written where the reference's plotter
    looks for it; returns the section."""
    sec = sectionCut(grid, plane, cut_index, rho_nominal_phys, soundspeed_phys)
    write_section_cut(path, plot_number, sec)
    return sec


def exportHistoryData(history, current_iteration: int, path: str = "/dev/shm/historyData.bin"):
    """exportHistoryData (exportSectionCutPlot.h:994-1001): int32 count = iteration + 1,
    then that many float32 history values."""
    count = int(current_iteration) + 1
    with open(path, "wb") as fh:
        np.array([count], dtype=np.int32).tofile(fh)
        np.asarray(history, dtype=np.float32)[:count].tofile(fh)


def drag_coefficient(drag_lattice: float, grid_info: InfoStruct, case: SphereCase, coarse_res: float = 1.0) -> float:
    """Cd = F / (rho U^2 pi D^2 / 8) with F and U in the units of the grid the force was
    summed on (the reference converts both to physical units: the factors cancel)."""
    # lattice units of a grid with cell size res: length unit res, time unit dt = res^2
    # scaled with nu fixed (acoustic scaling dt ~ res): U_grid = u_in * (res_coarse/res) *
    # (dt/dt_coarse) = u_in for 2:1 refinement; D_grid = D / res.
    d_cells = 2.0 * case.radius / grid_info.res
    return -8.0 * drag_lattice / (case.rho_given * case.u_in ** 2 * np.pi * d_cells ** 2)


def debug_cells(op: int, a0: int, f: np.ndarray, args: np.ndarray) -> np.ndarray:
    """Run one device function per row of `f` on the GPU (see psl_debug_cells)."""
    f = np.ascontiguousarray(f, dtype=np.float32).reshape(-1, 27).copy()
    args = np.ascontiguousarray(args, dtype=np.float32).reshape(-1, 4)
    assert args.shape[0] == f.shape[0]
    call("psl_debug_cells", op, a0, f.ctypes.data, args.ctypes.data, f.shape[0])
    return f
