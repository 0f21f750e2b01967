"""Flow-past-sphere configurations: grid metadata, hooks and start state.

* ``config1``: 128x64x64 single grid, sphere D=16 at (32,32,32), u_in=0.05, nu=0.008
  (Re=100), no LES, free-slip y/z walls, velocity inlet at x=0, pressure outlet at x=127.
* ``config2``: 512x256x256 coarse grid with one 2:1 refinement level over the coarse block
  [80,208) x [80,176) x [80,176) (128x96x96 coarse cells -> 256x192x192 fine cells),
  sphere D=48 at (128,128,128), Re=1e5 (nu_coarse = 0.05*48/1e5 = 2.4e-5, nu_fine = 2 nu),
  Smagorinsky C_s=0.1, same boundary conditions.

Both start from feq(rho=1, u_in + U(+-1e-4)) with a seeded counter-based noise.  Lengths
are in coarse-cell units (res=1 on the coarse grid).
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

from .grid import GridStruct, InfoStruct, SphereCase, fillEquilibriumFromFunction, setSmagorinskyConstant, setSphereCase


@dataclass(frozen=True)
class SphereConfig:
    name: str
    nx: int
    ny: int
    nz: int
    sphere: tuple
    radius: float
    u_in: float
    nu: float
    smagorinsky: float = 0.0
    wall_mode: int = 0
    seed: int = 1234
    noise: float = 1e-4
    refine: tuple | None = None  # ((i0, j0, k0), (i1, j1, k1)) coarse block, half-open
    refine2: tuple | None = None  # a third level: block on the level-1 grid (its own cells)
    cs_mode: int = 0  # 0 uniform C_s; 1 outlet sponge on the coarse grid (sponge_smagorinsky)

    def case(self) -> SphereCase:
        return SphereCase(sphere=tuple(float(v) for v in self.sphere), radius=float(self.radius), u_in=self.u_in,
                          rho_given=1.0, wall_mode=self.wall_mode, smagorinsky=self.smagorinsky, seed=self.seed,
                          noise=self.noise)

    def infos(self) -> list:
        c = InfoStruct(gridID=0, res=1.0, cellCountX=self.nx, cellCountY=self.ny, cellCountZ=self.nz, nu=self.nu)
        out = [c]
        if self.refine:
            (c.iSubgridStart, c.jSubgridStart, c.kSubgridStart), (c.iSubgridEnd, c.jSubgridEnd, c.kSubgridEnd) = self.refine
            f = c.finer()
            out.append(f)
            if self.refine2:
                (f.iSubgridStart, f.jSubgridStart, f.kSubgridStart), (f.iSubgridEnd, f.jSubgridEnd, f.kSubgridEnd) = \
                    self.refine2
                out.append(f.finer())
        return out

    def updates_per_step(self) -> int:
        """Cells actually updated per coarse step: on every level the cells that are neither
        in the fine grids' one-cell ghost layer nor in a refined interior
        (include/applyLocalCellUpdate.h:25-30), times the level's 2^level sub-steps."""
        total = 0
        for level, info in enumerate(self.infos()):
            nx, ny, nz = info.cellCountX, info.cellCountY, info.cellCountZ
            cells = nx * ny * nz if level == 0 else (nx - 2) * (ny - 2) * (nz - 2)
            if info.iSubgridEnd > info.iSubgridStart:
                cells -= (max(0, info.iSubgridEnd - info.iSubgridStart - 4) *
                          max(0, info.jSubgridEnd - info.jSubgridStart - 4) *
                          max(0, info.kSubgridEnd - info.kSubgridStart - 4))
            total += cells * 2 ** level
        return total

    def reference_updates_per_step(self) -> int:
        """The reference driver's own count (flowAroundSphereMainSingle.cu:225-234), which
        subtracts (n-2)^3 per refined block instead of the (n-4)^3 cells it skips and
        counts the fine ghost layer."""
        n = self.nx * self.ny * self.nz
        if not self.refine:
            return n
        (i0, j0, k0), (i1, j1, k1) = self.refine
        fx, fy, fz = 2 * (i1 - i0), 2 * (j1 - j0), 2 * (k1 - k0)
        return n - (i1 - i0 - 2) * (j1 - j0 - 2) * (k1 - k0 - 2) + 2 * fx * fy * fz


def config1(**kw) -> SphereConfig:
    c = SphereConfig(name="sphere_128x64x64_re100", nx=128, ny=64, nz=64, sphere=(32.0, 32.0, 32.0), radius=8.0,
                     u_in=0.05, nu=0.05 * 16 / 100)
    return replace(c, **kw)


def config2(scale: float = 1.0, **kw) -> SphereConfig:
    """`scale` shrinks every length (grid, sphere, block) for small profiling runs; the
    Reynolds number is kept (nu scales with the diameter)."""
    def s(v):
        return int(round(v * scale))

    name = "sphere_512x256x256_re1e5_refined" if scale == 1.0 else f"sphere_{s(512)}x{s(256)}x{s(256)}_re1e5_refined"
    c = SphereConfig(name=name, nx=s(512), ny=s(256), nz=s(256), sphere=(128.0 * scale,) * 3,
                     radius=24.0 * scale, u_in=0.05, nu=0.05 * 48 * scale / 1e5, smagorinsky=0.1,
                     refine=((s(80), s(80), s(80)), (s(208), s(176), s(176))))
    return replace(c, **kw)


def sponge_smagorinsky(info: InfoStruct, cs: float) -> np.ndarray:
    """getSmagorinskyConstant(i, j, k, Info) of a sponge layer ahead of the outlet, for every
    cell of a grid in cell order: C_s rises linearly from `cs` at i = 3 Nx / 4 to 4 cs at
    the outlet plane.  Evaluated in FP32 with one rounding per operation, in the order of
    the C++ hook cs * (1 + 3 (i - i0) / (Nx - 1 - i0)), so both give the same numbers."""
    nx, ny, nz = info.cellCountX, info.cellCountY, info.cellCountZ
    i0 = (3 * nx) // 4
    i = np.arange(nx)
    ramp = np.float32(3.0) * (i - i0).astype(np.float32)
    ramp = ramp / np.float32(nx - 1 - i0)
    row = np.where(i > i0, np.float32(cs) * (np.float32(1.0) + ramp), np.float32(cs)).astype(np.float32)
    return np.broadcast_to(row, (nz, ny, nx)).reshape(-1).copy()


def make_sphere_grids(cfg: SphereConfig, storage: str = "f32", one_mapping: bool = False) -> tuple:
    """Allocate the grids of `cfg`, evaluate the case hooks into markers (and, for
    cs_mode 1, the coarse grid's per-cell Smagorinsky constants) and fill the start state.
    ``one_mapping``: population rows in one plain allocation (GridStruct).  Returns
    (grids, case)."""
    case = cfg.case()
    grids = []
    for info in cfg.infos():
        g = GridStruct(info, storage=storage, one_mapping=one_mapping)
        setSphereCase(g, case)
        if cfg.cs_mode == 1 and info.gridID == 0:
            setSmagorinskyConstant(g, sponge_smagorinsky(info, cfg.smagorinsky))
        fillEquilibriumFromFunction(g, case)
        grids.append(g)
    return grids, case
