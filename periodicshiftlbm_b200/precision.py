"""Precision study of the storage forms: FP32, FP16 and BF16 (f - w shifted) population
storage, each against an FP64-storage, FP64-arithmetic run of the same case.

For each form the study runs the refined flow-past-sphere case for `steps` coarse steps and
reports
  * the relative L2 error of the velocity magnitude |u| at the last step, over every cell
    that the update touches on every level (not solid, not skipped), against the FP64 run;
  * the sphere drag (momentum exchange, FP64 reduction, on the finest level) and drag
    coefficient at the last step and averaged over the sampled last `average_last` fraction
    of the run (default one fifth), and their relative errors against the FP64 run.

The wake is unsteady: runs that differ in rounding drift apart in shedding phase, so the
drag at one step differs by several percent between any two forms, FP32 against FP64
included, and a mean is comparable only over several shedding periods.

A form "<storage>+mlp" runs that storage with the learned closure (the packaged weights,
periodicshiftlbm_b200/data) in place of Smagorinsky; its errors against the FP64
(Smagorinsky) run then hold the model difference as well as the rounding.  "<storage>+mlpK"
(16-bit storage) runs the closure's network on every K-th update only, each cell relaxing
with its kept nu_t in between (psl_set_sgs_mlp_interval).

``python -m periodicshiftlbm_b200.precision --scale 0.5 --steps 5000`` runs the
256x128x128 two-level subsample of the 512x256x256 Re=1e5 sphere case.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import _lib
from .cases import SphereConfig, config2, make_sphere_grids
from .grid import drag_coefficient, getSphereDrag, updateGrid


def flow_cells(grid) -> np.ndarray:
    """Cells the update kernel collides: every marker kind except skip and solid."""
    kind = grid.markers & 7
    return (kind != _lib.CELL_SKIP) & (kind != _lib.CELL_SOLID)


def updated_cells(grid) -> np.ndarray:
    """Cells the update kernel writes (solid cells are bounced back, skip cells untouched)."""
    return (grid.markers & 7) != _lib.CELL_SKIP


def speed(grids) -> np.ndarray:
    """|u| over the flow cells of every level, concatenated level by level (FP64)."""
    out = []
    for g in grids:
        m = g.macroscopic()
        sel = flow_cells(g)
        out.append(np.sqrt(m[1, sel] ** 2 + m[2, sel] ** 2 + m[3, sel] ** 2))
    return np.concatenate(out)


def speed_error(grids, ref_grids) -> float:
    """Relative L2 error of |u| of `grids` against `ref_grids` (same case, same cells)."""
    a, b = speed(grids), speed(ref_grids)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run_form(cfg: SphereConfig, storage: str, steps: int, sample_every: int = 50, average_last: float = 0.2):
    """Run `cfg` in one storage form; returns (grids, result dict).  The caller closes the
    grids."""
    storage, _, closure = storage.partition("+")
    grids, case = make_sphere_grids(cfg, storage=storage)
    if closure.startswith("mlp"):
        from .sgs import load_params, set_sgs_mlp

        params = load_params()
        interval = int(closure[3:] or 1)
        for g in grids:
            set_sgs_mlp(g, params, g.Info.res / grids[0].Info.res, interval=interval if interval > 1 else None)
    fine = grids[-1]
    drags = []
    t0 = time.perf_counter()
    for s in range(1, steps + 1):
        updateGrid(grids, 0)
        if s % sample_every == 0 and s > steps - int(steps * average_last):
            drags.append(getSphereDrag(fine, case))
    last = getSphereDrag(fine, case)
    elapsed = time.perf_counter() - t0
    health = [g.health() for g in grids]
    mean = float(np.mean(drags)) if drags else last
    return grids, {
        "storage": storage + ("+" + closure if closure else ""),
        "steps": steps,
        "drag_last": last,
        "average_last": average_last,
        "drag_mean": mean,
        "cd_last": drag_coefficient(last, fine.Info, case),
        "cd_mean": drag_coefficient(mean, fine.Info, case),
        "health": health,
        "seconds": elapsed,
    }


def study(cfg: SphereConfig, steps: int, forms=("f32", "f16", "bf16"), sample_every: int = 50,
          average_last: float = 0.2) -> dict:
    ref_grids, ref = run_form(cfg, "f64", steps, sample_every, average_last)
    ref_speed = speed(ref_grids)
    for g in ref_grids:
        g.close()
    out = {"case": cfg.name, "steps": steps, "f64": ref, "forms": {}}
    for s in forms:
        grids, r = run_form(cfg, s, steps, sample_every, average_last)
        a = speed(grids)
        r["speed_l2_rel_error"] = float(np.linalg.norm(a - ref_speed) / np.linalg.norm(ref_speed))
        r["drag_rel_error_last"] = abs(r["drag_last"] - ref["drag_last"]) / abs(ref["drag_last"])
        r["drag_rel_error_mean"] = abs(r["drag_mean"] - ref["drag_mean"]) / abs(ref["drag_mean"])
        out["forms"][s] = r
        for g in grids:
            g.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--scale", type=float, default=0.5)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--sample-every", type=int, default=50)
    ap.add_argument("--forms", default="f32,f16,bf16")
    ap.add_argument("--average-last", type=float, default=0.2, help="fraction of the run the drag mean covers")
    a = ap.parse_args(argv)
    res = study(config2(a.scale), a.steps, tuple(a.forms.split(",")), a.sample_every, a.average_last)
    print(json.dumps({"command": "python -m periodicshiftlbm_b200.precision " + " ".join(argv or sys.argv[1:]), **res}))


if __name__ == "__main__":
    main()
