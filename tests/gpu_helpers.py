"""Shared helpers for the GPU tests: run an oracle-described sphere case through the CUDA
library's public API."""
import numpy as np

from periodicshiftlbm_b200 import updateGrid
from periodicshiftlbm_b200.cases import SphereConfig, make_sphere_grids


def config_from_case(case) -> SphereConfig:
    """oracle.bindings.SphereCase -> the package's SphereConfig (same fields)."""
    return SphereConfig(name="test", nx=case.nx, ny=case.ny, nz=case.nz, sphere=tuple(case.sphere),
                        radius=case.radius, u_in=case.u_in, nu=case.nu, smagorinsky=case.smagorinsky,
                        wall_mode=case.wall_mode, seed=case.seed, noise=case.noise, refine=case.refine,
                        refine2=case.refine2, cs_mode=case.cs_mode)


class GpuSim:
    def __init__(self, case, storage="f32"):
        self.cfg = config_from_case(case)
        self.grids, self.sc = make_sphere_grids(self.cfg, storage=storage)
        self.levels = len(self.grids)

    def run(self, steps):
        for _ in range(steps):
            updateGrid(self.grids, 0)

    def populations(self, level=0):
        return self.grids[level].fArray

    def shifts(self, level=0):
        return self.grids[level].shifter

    def drag(self):
        from periodicshiftlbm_b200 import getSphereDrag

        return getSphereDrag(self.grids[-1], self.sc)

    def close(self):
        for g in self.grids:
            g.close()


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)))


def l2rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
