"""Batched form: many independent flow-past-sphere cases of uneven grid size and Reynolds
number advanced by one persistent kernel per step, replayed from a captured CUDA graph,
with the launch shape chosen by the library's autotuner (include/psl.h, psl_batch_*).

``batch_configs`` draws the seeded case set of the batched benchmark: x-extent in
{64, 96, 128, 192}, y = z = x/2, sphere diameter x/8 centred at (x/4, y/2, z/2), Reynolds
number log-uniform in [1e2, 1e6] (nu = u_in D / Re), Smagorinsky C_s = 0.1 when Re > 1e3,
FP32 populations, the boundary conditions and noisy equilibrium start of the sphere cases.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PslBatchTuning, call
from .cases import SphereConfig, make_sphere_grids

X_EXTENTS = (64, 96, 128, 192)


def batch_configs(count: int = 64, seed: int = 2024, u_in: float = 0.05) -> list:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        x = int(rng.choice(X_EXTENTS))
        y = x // 2
        d = x / 8.0
        re = float(10.0 ** rng.uniform(2.0, 6.0))
        out.append(SphereConfig(name=f"batch{i}_{x}x{y}x{y}_re{re:.3g}", nx=x, ny=y, nz=y,
                                sphere=(x / 4.0, y / 2.0, y / 2.0), radius=d / 2.0, u_in=u_in, nu=u_in * d / re,
                                smagorinsky=0.1 if re > 1e3 else 0.0, seed=1000 + i))
    return out


def make_batch_grids(configs, storage: str = "f32"):
    """One single-level grid per config (markers and start state filled).  Returns
    (grids, cases)."""
    grids, cases = [], []
    for cfg in configs:
        g, c = make_sphere_grids(cfg, storage=storage)
        assert len(g) == 1, "batched cases are single-level"
        grids.append(g[0])
        cases.append(c)
    return grids, cases


class Batch:
    """A psl_batch over `grids` (kept alive by this object)."""

    def __init__(self, grids):
        self.grids = list(grids)
        arr = (ctypes.c_void_p * len(self.grids))(*[g.handle.value for g in self.grids])
        self._h = ctypes.c_void_p()
        call("psl_batch_create", arr, len(self.grids), ctypes.byref(self._h))

    def close(self):
        if self._h and self._h.value:
            _lib.lib().psl_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, steps: int):
        call("psl_batch_run", self._h, int(steps))

    def synchronize(self):
        call("psl_batch_synchronize", self._h)

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        call("psl_batch_get_stream", self._h, ctypes.byref(s))
        return s.value or 0

    @property
    def tuning(self) -> dict:
        t = PslBatchTuning()
        call("psl_batch_get_tuning", self._h, ctypes.byref(t))
        return {"threads": t.threads, "tile_cells": t.tile_cells, "blocks_per_sm": t.blocks_per_sm,
                "ms_per_step": t.ms_per_step}

    @tuning.setter
    def tuning(self, d: dict):
        t = PslBatchTuning(int(d["threads"]), int(d["tile_cells"]), int(d["blocks_per_sm"]), 0.0)
        call("psl_batch_set_tuning", self._h, ctypes.byref(t))

    def autotune(self, trial_steps: int = 5) -> dict:
        t = PslBatchTuning()
        call("psl_batch_autotune", self._h, int(trial_steps), ctypes.byref(t))
        return self.tuning

    def cells(self) -> int:
        return sum(g.cellCount for g in self.grids)


def study(count: int = 64, steps: int = 2000, seed: int = 2024, trial_steps: int = 3) -> dict:
    """Run the seeded case set batched and each case solo for `steps` steps; report the
    batched throughput, the autotuner's choice and the per-case drag of both runs."""
    import time

    from .grid import drag_coefficient, getSphereDrag, updateGrid

    configs = batch_configs(count, seed)
    grids, cases = make_batch_grids(configs)
    b = Batch(grids)
    tuning = b.autotune(trial_steps)
    b.run(1)  # capture + first replay
    b.synchronize()
    t0 = time.perf_counter()
    b.run(steps - 1)
    b.synchronize()
    wall = time.perf_counter() - t0
    batched = [getSphereDrag(g, c) for g, c in zip(grids, cases)]
    cells = b.cells()
    b.close()
    for g in grids:
        g.close()
    rows = []
    for cfg, drag_b in zip(configs, batched):
        solo, case = make_sphere_grids(cfg)
        for _ in range(steps):
            updateGrid(solo, 0)
        drag_s = getSphereDrag(solo[0], case)
        rows.append({"case": cfg.name, "cells": cfg.nx * cfg.ny * cfg.nz, "re": 0.05 * 2 * cfg.radius / cfg.nu,
                     "drag_batched": drag_b, "drag_solo": drag_s,
                     "cd_batched": drag_coefficient(drag_b, solo[0].Info, case),
                     "rel_diff": abs(drag_b - drag_s) / max(abs(drag_s), 1e-30)})
        solo[0].close()
    return {"cases": count, "steps": steps, "total_cells": cells, "tuning": tuning,
            "wall_mlups_after_first_step": cells * (steps - 1) / wall / 1e6, "per_case": rows,
            "max_rel_drag_diff": max(r["rel_diff"] for r in rows)}


def main(argv=None):
    import argparse
    import json

    ap = argparse.ArgumentParser(description="batched sphere cases vs solo runs")
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args(argv)
    print(json.dumps(study(a.cases, a.steps, a.seed)))


if __name__ == "__main__":
    main()
