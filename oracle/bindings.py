"""ctypes bindings for the two CPU checkers built by oracle/Makefile.

ORACLE / TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, never by the product package.

* ``RefLib``   -- oracle/_ref/libpsl_ref.so: the reference project's own headers compiled
  unmodified for the host (see oracle/ref_cases.cpp).
* ``OracleLib`` -- oracle/liboracle.so: the project's own C++ restatement (float/double).

Both expose the same case description (``CaseConfig``) so a test can run one sphere
configuration through the reference, the restatement and the CUDA path.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libpsl_ref.so")
ORACLE_SO = os.path.join(HERE, "liboracle.so")


class CaseConfig(ctypes.Structure):
    """Mirrors ``RefCaseConfig`` in oracle/ref_cases.cpp and ``OracleCaseConfig``."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("levels", ctypes.c_int),
        ("iSub0", ctypes.c_int), ("jSub0", ctypes.c_int), ("kSub0", ctypes.c_int),
        ("iSub1", ctypes.c_int), ("jSub1", ctypes.c_int), ("kSub1", ctypes.c_int),
        ("sphereX", ctypes.c_float), ("sphereY", ctypes.c_float), ("sphereZ", ctypes.c_float),
        ("sphereR", ctypes.c_float),
        ("uIn", ctypes.c_float),
        ("nuCoarse", ctypes.c_float),
        ("smagorinsky", ctypes.c_float),
        ("wallMode", ctypes.c_int),
        ("seed", ctypes.c_uint32),
        ("noiseAmp", ctypes.c_float),
        ("iSub2_0", ctypes.c_int), ("jSub2_0", ctypes.c_int), ("kSub2_0", ctypes.c_int),
        ("iSub2_1", ctypes.c_int), ("jSub2_1", ctypes.c_int), ("kSub2_1", ctypes.c_int),
        ("csMode", ctypes.c_int),
        ("forceR0", ctypes.c_float), ("forceR1", ctypes.c_float), ("forceOmega", ctypes.c_float),
    ]


@dataclass
class SphereCase:
    """Flow past a sphere in a channel (coarse-cell units)."""

    nx: int = 128
    ny: int = 64
    nz: int = 64
    sphere: tuple = (32.0, 32.0, 32.0)
    radius: float = 8.0
    u_in: float = 0.05
    nu: float = 0.008
    smagorinsky: float = 0.0
    wall_mode: int = 0  # 0 free-slip mirror walls, 1 velocity walls (reference driver scheme)
    seed: int = 1234
    noise: float = 1e-4
    refine: tuple | None = None  # ((i0, j0, k0), (i1, j1, k1)) coarse block, half-open
    refine2: tuple | None = None  # a third level: block on the level-1 grid (its own cells)
    cs_mode: int = 0  # 0 uniform Smagorinsky constant, 1 outlet sponge (getSmagorinskyConstant per cell)
    force_annulus: tuple | None = None  # (R0, R1, omega): forced-velocity cells for getTorque (reference build)

    def to_ctypes(self) -> CaseConfig:
        c = CaseConfig()
        c.nx, c.ny, c.nz = self.nx, self.ny, self.nz
        c.levels = (3 if self.refine2 else 2) if self.refine else 1
        if self.refine:
            (c.iSub0, c.jSub0, c.kSub0), (c.iSub1, c.jSub1, c.kSub1) = self.refine
        if self.refine2:
            (c.iSub2_0, c.jSub2_0, c.kSub2_0), (c.iSub2_1, c.jSub2_1, c.kSub2_1) = self.refine2
        c.sphereX, c.sphereY, c.sphereZ = self.sphere
        c.sphereR = self.radius
        c.uIn = self.u_in
        c.nuCoarse = self.nu
        c.smagorinsky = self.smagorinsky
        c.wallMode = self.wall_mode
        c.seed = self.seed
        c.noiseAmp = self.noise
        c.csMode = self.cs_mode
        if self.force_annulus:
            c.forceR0, c.forceR1, c.forceOmega = self.force_annulus
        return c


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class _SimLib:
    prefix = ""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
        self.lib = ctypes.CDLL(path)
        p = self.prefix
        L = self.lib
        getattr(L, p + "sim_create").restype = ctypes.c_void_p
        getattr(L, p + "sim_create").argtypes = [ctypes.POINTER(CaseConfig)]
        getattr(L, p + "sim_destroy").argtypes = [ctypes.c_void_p]
        getattr(L, p + "sim_run").argtypes = [ctypes.c_void_p, ctypes.c_int]
        getattr(L, p + "sim_cell_count").restype = ctypes.c_longlong
        getattr(L, p + "sim_cell_count").argtypes = [ctypes.c_void_p, ctypes.c_int]
        getattr(L, p + "sim_get_f").argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        getattr(L, p + "sim_set_f").argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        getattr(L, p + "sim_get_shifts").argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        getattr(L, p + "sim_drag").restype = ctypes.c_double
        getattr(L, p + "sim_drag").argtypes = [ctypes.c_void_p]
        getattr(L, p + "sim_fill_coarse_from_fine").argtypes = [ctypes.c_void_p, ctypes.c_int]

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)


class Sim:
    """A running case on one of the CPU checkers."""

    def __init__(self, owner: _SimLib, case: SphereCase, **kw):
        self.owner = owner
        self.case = case
        self.cfg = case.to_ctypes()
        self.h = owner._create(self.cfg, **kw)
        self.levels = self.cfg.levels

    def close(self):
        if self.h:
            self.owner._fn("sim_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, steps: int):
        self.owner._fn("sim_run")(self.h, int(steps))

    def cell_count(self, level: int = 0) -> int:
        return int(self.owner._fn("sim_cell_count")(self.h, level))

    def populations(self, level: int = 0) -> np.ndarray:
        n = self.cell_count(level)
        out = np.empty((27, n), dtype=getattr(self, "dtype", self.owner.dtype))
        self.owner._fn("sim_get_f")(self.h, level, out.ctypes.data)
        return out

    def set_populations(self, f: np.ndarray, level: int = 0):
        f = np.ascontiguousarray(f, dtype=getattr(self, "dtype", self.owner.dtype))
        self.owner._fn("sim_set_f")(self.h, level, f.ctypes.data)

    def shifts(self, level: int = 0) -> np.ndarray:
        out = np.zeros(27, dtype=np.int32)
        self.owner._fn("sim_get_shifts")(self.h, level, out.ctypes.data)
        return out

    def drag(self) -> float:
        return float(self.owner._fn("sim_drag")(self.h))

    def fill_coarse_from_fine(self, level: int = 0):
        """fillCoarseGridFromFine on levels `level` and `level` + 1."""
        self.owner._fn("sim_fill_coarse_from_fine")(self.h, int(level))

    def torque(self, level: int = 0) -> float:
        """The reference's getTorque written for PS grids (reference build only)."""
        return float(self.owner.lib.ref_sim_torque(self.h, level))

    def flow_report(self, level: int, plane: str, cut_index: int, bounds6) -> dict:
        """The reference's getFlowReportGeneral over this level alone, as a one-level DIAD
        grid holding the level's state (reference build only)."""
        planes = {"XY": 0, "ZY": 1, "ZX": 2}
        b = np.ascontiguousarray(bounds6, dtype=np.float32)
        out = np.zeros(5, dtype=np.float32)
        self.owner.lib.ref_sim_flow_report_single(self.h, level, planes[plane], cut_index, b.ctypes.data,
                                                  out.ctypes.data)
        return {"ux": float(out[0]), "uy": float(out[1]), "uz": float(out[2]), "rho": float(out[3]),
                "area": float(out[4])}

    def export_section(self, level: int, plane: str, cut_index: int, plot_number: int, path: str):
        """The reference's exportSectionCutPlotGeneral of one level, written to `path`
        (reference build only)."""
        planes = {"XY": 0, "ZY": 1, "ZX": 2}
        self.owner.lib.ref_sim_export_section(self.h, level, planes[plane], cut_index, plot_number, path.encode())


class RefLib(_SimLib):
    """The reference's own code (compiled through the TNL shim)."""

    prefix = "ref_"
    dtype = np.float32

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        L = self.lib
        f = ctypes.c_float
        i = ctypes.c_int
        vp = ctypes.c_void_p
        L.ref_collision.argtypes = [vp, f, f]
        L.ref_feq.argtypes = [f, f, f, f, vp]
        L.ref_rho_u.argtypes = [vp, vp]
        L.ref_omega_les.argtypes = [vp, f, f, vp]
        L.ref_mbbc.argtypes = [i, i, i, f, f, f, f, vp]
        L.ref_restore_rho.argtypes = [i, i, i, f, f, f, vp, vp]
        L.ref_restore_u.argtypes = [i, i, i, f, vp, vp]
        L.ref_restore_rho_u.argtypes = [i, i, i, vp, vp]
        L.ref_mirror.argtypes = [i, i, i, vp]
        L.ref_bounceback.argtypes = [vp]
        L.ref_moving_bounceback.argtypes = [vp, f, f, f]
        L.ref_scalar_collision.argtypes = [vp, vp, f]
        L.ref_sim_enable_scalar.argtypes = [vp, f, ctypes.c_int]
        L.ref_sim_set_T.argtypes = [vp, vp]
        L.ref_sim_get_T.argtypes = [vp, vp]
        L.ref_rescale.argtypes = [vp, i]
        L.ref_streaming.argtypes = [i, i, i, vp]
        L.ref_smagorinsky_constants.argtypes = [ctypes.POINTER(CaseConfig), i, i, i, i, vp]
        L.ref_sim_export_section.argtypes = [vp, i, i, i, i, ctypes.c_char_p]
        L.ref_sim_torque.argtypes = [vp, i]
        L.ref_sim_torque.restype = f
        L.ref_sim_flow_report_single.argtypes = [vp, i, i, i, vp, vp]
        L.ref_export_history.argtypes = [vp, i, i, ctypes.c_char_p]
        for n in ("ref_sim_periodic_x", "ref_sim_periodic_y", "ref_sim_streaming"):
            getattr(L, n).argtypes = [vp, i]

    def _create(self, cfg, **kw):
        return self.lib.ref_sim_create(ctypes.byref(cfg))

    def export_history(self, values, current_iteration: int, path: str):
        """exportHistoryData of the reference, written to `path`."""
        v = np.ascontiguousarray(values, dtype=np.float32)
        self.lib.ref_export_history(v.ctypes.data, v.size, current_iteration, path.encode())

    def smagorinsky_constants(self, case: SphereCase, grid_id: int, nx: int, ny: int, nz: int) -> np.ndarray:
        """The case's getSmagorinskyConstant hook over every cell of a grid (cell order)."""
        out = np.zeros(nx * ny * nz, dtype=np.float32)
        cfg = case.to_ctypes()
        self.lib.ref_smagorinsky_constants(ctypes.byref(cfg), grid_id, nx, ny, nz, out.ctypes.data)
        return out

    def sim(self, case: SphereCase) -> Sim:
        return Sim(self, case)

    # ---- single-function pins (float32 arrays of 27) ----
    def collision(self, f, nu, cs):
        a = np.array(f, dtype=np.float32)
        self.lib.ref_collision(a.ctypes.data, nu, cs)
        return a

    def feq(self, rho, ux, uy, uz):
        a = np.zeros(27, dtype=np.float32)
        self.lib.ref_feq(rho, ux, uy, uz, a.ctypes.data)
        return a

    def rho_u(self, f):
        a = np.array(f, dtype=np.float32)
        o = np.zeros(4, dtype=np.float32)
        self.lib.ref_rho_u(a.ctypes.data, o.ctypes.data)
        return o

    def omega_les(self, f, nu, cs):
        a = np.array(f, dtype=np.float32)
        o = np.zeros(1, dtype=np.float32)
        self.lib.ref_omega_les(a.ctypes.data, nu, cs, o.ctypes.data)
        return float(o[0])

    def mbbc(self, n, rho, ux, uy, uz, f):
        a = np.array(f, dtype=np.float32)
        self.lib.ref_mbbc(n[0], n[1], n[2], rho, ux, uy, uz, a.ctypes.data)
        return a

    def restore_rho(self, n, ux, uy, uz, f, rho0=1.0):
        a = np.array(f, dtype=np.float32)
        o = np.array([rho0], dtype=np.float32)
        self.lib.ref_restore_rho(n[0], n[1], n[2], ux, uy, uz, a.ctypes.data, o.ctypes.data)
        return float(o[0])

    def restore_u(self, n, rho, f, u0=(0.0, 0.0, 0.0)):
        a = np.array(f, dtype=np.float32)
        o = np.array(u0, dtype=np.float32)
        self.lib.ref_restore_u(n[0], n[1], n[2], rho, a.ctypes.data, o.ctypes.data)
        return o

    def restore_rho_u(self, n, f, init=(1.0, 0.0, 0.0, 0.0)):
        a = np.array(f, dtype=np.float32)
        o = np.array(init, dtype=np.float32)
        self.lib.ref_restore_rho_u(n[0], n[1], n[2], a.ctypes.data, o.ctypes.data)
        return o

    def mirror(self, n, f):
        a = np.array(f, dtype=np.float32)
        self.lib.ref_mirror(n[0], n[1], n[2], a.ctypes.data)
        return a

    def bounceback(self, f):
        a = np.array(f, dtype=np.float32)
        self.lib.ref_bounceback(a.ctypes.data)
        return a

    def moving_bounceback(self, f, ux, uy, uz):
        a = np.array(f, dtype=np.float32)
        self.lib.ref_moving_bounceback(a.ctypes.data, ux, uy, uz)
        return a

    def scalar_collision(self, f, T, tauT):
        a = np.array(f, dtype=np.float32)
        t = np.array(T, dtype=np.float32)
        self.lib.ref_scalar_collision(a.ctypes.data, t.ctypes.data, tauT)
        return t

    def enable_scalar(self, sim, tauT: float, inlet: bool):
        """The reference's scalar-transport update on grid 0 of `sim` (T starts at 0); with
        `inlet`, concentration 1 is prescribed on the lower half (j < Ny/2) of the inlet
        plane and 0 on the upper half."""
        self.lib.ref_sim_enable_scalar(sim.h, tauT, 1 if inlet else 0)

    def scalar_populations(self, sim):
        out = np.empty((27, sim.cell_count(0)), dtype=np.float32)
        self.lib.ref_sim_get_T(sim.h, out.ctypes.data)
        return out

    def set_scalar_populations(self, sim, t):
        t = np.ascontiguousarray(t, dtype=np.float32)
        self.lib.ref_sim_set_T(sim.h, t.ctypes.data)

    def rescale(self, f, coarse_to_fine: bool):
        a = np.array(f, dtype=np.float32)
        self.lib.ref_rescale(a.ctypes.data, 1 if coarse_to_fine else 0)
        return a

    def streaming(self, dims, shifts):
        s = np.array(shifts, dtype=np.int32)
        self.lib.ref_streaming(dims[0], dims[1], dims[2], s.ctypes.data)
        return s


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class OracleLib(_SimLib):
    """The project's own C++ restatement (oracle/psl_oracle.cpp), float or double."""

    prefix = "oracle_"

    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path)
        L = self.lib
        getattr(L, "oracle_sim_create").argtypes = [ctypes.POINTER(CaseConfig), ctypes.c_int]
        vp = ctypes.c_void_p
        i = ctypes.c_int
        for suf, T in (("f32", ctypes.c_float), ("f64", ctypes.c_double)):
            g = lambda n: getattr(L, f"oracle_{n}_{suf}")  # noqa: E731
            g("collision").argtypes = [vp, T, T]
            g("collision_forced").argtypes = [vp, T, T, T, T, T]
            g("feq").argtypes = [T, T, T, T, vp]
            g("rescale").argtypes = [vp, i]
            g("mbbc").argtypes = [i, T, T, T, T, vp]
            g("restore_rho").argtypes = [i, T, T, T, vp, vp]
            g("restore_u").argtypes = [i, T, vp, vp]
            g("restore_rho_u").argtypes = [i, vp, vp]
            g("mirror").argtypes = [i, vp]
            g("bounceback").argtypes = [vp]
            g("moving_bounceback").argtypes = [vp, T, T, T]
            g("omega_les").argtypes = [vp, T, T]
            g("omega_les").restype = T
        L.oracle_streaming.argtypes = [i, i, i, vp]

    def _create(self, cfg, double=False):
        return self.lib.oracle_sim_create(ctypes.byref(cfg), 1 if double else 0)

    def sim(self, case: SphereCase, double: bool = False) -> Sim:
        s = Sim.__new__(Sim)
        s.owner = self
        s.case = case
        s.cfg = case.to_ctypes()
        s.levels = s.cfg.levels
        s.dtype = np.float64 if double else np.float32
        s.h = self._create(s.cfg, double=double)
        return s

    @property
    def dtype(self):  # per-sim dtype; see OracleSim
        return np.float32

    def _fn1(self, name, dtype):
        return getattr(self.lib, f"oracle_{name}_{'f64' if dtype == np.float64 else 'f32'}")

    @staticmethod
    def normal_index(n):
        return (n[0] + 1) * 9 + (n[1] + 1) * 3 + (n[2] + 1)

    def collision(self, f, nu, cs, dtype=np.float32, force=None):
        a = np.array(f, dtype=dtype)
        if force is None:
            self._fn1("collision", dtype)(a.ctypes.data, nu, cs)
        else:
            self._fn1("collision_forced", dtype)(a.ctypes.data, nu, cs, *force)
        return a

    def feq(self, rho, ux, uy, uz, dtype=np.float32):
        a = np.zeros(27, dtype=dtype)
        self._fn1("feq", dtype)(rho, ux, uy, uz, a.ctypes.data)
        return a

    def rescale(self, f, coarse_to_fine, dtype=np.float32):
        a = np.array(f, dtype=dtype)
        self._fn1("rescale", dtype)(a.ctypes.data, 1 if coarse_to_fine else 0)
        return a

    def mbbc(self, n, rho, ux, uy, uz, f, dtype=np.float32):
        a = np.array(f, dtype=dtype)
        self._fn1("mbbc", dtype)(self.normal_index(n), rho, ux, uy, uz, a.ctypes.data)
        return a

    def restore_rho(self, n, ux, uy, uz, f, rho0=1.0, dtype=np.float32):
        a = np.array(f, dtype=dtype)
        o = np.array([rho0], dtype=dtype)
        self._fn1("restore_rho", dtype)(self.normal_index(n), ux, uy, uz, a.ctypes.data, o.ctypes.data)
        return float(o[0])

    def restore_u(self, n, rho, f, u0=(0.0, 0.0, 0.0), dtype=np.float32):
        a = np.array(f, dtype=dtype)
        o = np.array(u0, dtype=dtype)
        self._fn1("restore_u", dtype)(self.normal_index(n), rho, a.ctypes.data, o.ctypes.data)
        return o

    def restore_rho_u(self, n, f, init=(1.0, 0.0, 0.0, 0.0), dtype=np.float32):
        a = np.array(f, dtype=dtype)
        o = np.array(init, dtype=dtype)
        self._fn1("restore_rho_u", dtype)(self.normal_index(n), a.ctypes.data, o.ctypes.data)
        return o

    def mirror(self, n, f, dtype=np.float32):
        a = np.array(f, dtype=dtype)
        self._fn1("mirror", dtype)(self.normal_index(n), a.ctypes.data)
        return a

    def bounceback(self, f, dtype=np.float32):
        a = np.array(f, dtype=dtype)
        self._fn1("bounceback", dtype)(a.ctypes.data)
        return a

    def moving_bounceback(self, f, ux, uy, uz, dtype=np.float32):
        a = np.array(f, dtype=dtype)
        self._fn1("moving_bounceback", dtype)(a.ctypes.data, ux, uy, uz)
        return a

    def omega_les(self, f, nu, cs, dtype=np.float32):
        a = np.array(f, dtype=dtype)
        return float(self._fn1("omega_les", dtype)(a.ctypes.data, nu, cs))

    def streaming(self, dims, shifts):
        s = np.array(shifts, dtype=np.int32)
        self.lib.oracle_streaming(dims[0], dims[1], dims[2], s.ctypes.data)
        return s


def oracle_available() -> bool:
    return os.path.exists(ORACLE_SO)


ALL_NORMALS = [(x, y, z) for x in (-1, 0, 1) for y in (-1, 0, 1) for z in (-1, 0, 1) if (x, y, z) != (0, 0, 0)]
