"""Benchmark of the per-step lattice update on the flow-past-sphere workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--config 1|2]
                    [--storage f32|f16|bf16] [--form single|batch]

Workload (default): 512x256x256 FP32 D3Q27 grid with one 2:1 refinement level over a
128x96x96 coarse block (256x192x192 fine cells), sphere D=48 at (128,128,128), Re=1e5,
cumulant collision + Smagorinsky C_s=0.1, free-slip walls, velocity inlet, pressure
outlet.  One step = one coarse time step = updateGrid(grids, 0): coarse streaming +
update, two fine streaming + update, one coarse/fine transfer: 50,843,696 cell updates.
Inputs (3.62 GB coarse + 1.02 GB fine of FP32 populations) are larger than L2, so no L2
flush is needed.

`--form batch` measures the batched form instead: 64 seeded single-level sphere cases
(x in {64,96,128,192}, y=z=x/2, D=x/8, Re log-uniform in [1e2,1e6]) advanced by one
persistent kernel per step from a captured CUDA graph, launch shape from the autotuner.

Prints ONE JSON line (rank 0).  `value` is MLUPS over the device-timed region (CUDA events,
max over ranks); `e2e` is the same metric through the public API with host buffers: the
state is uploaded from pinned host memory, every step's FP64 drag is copied back to pinned
host memory in stream order (the reference driver reads it every step), at the end the
coarse levels are filled from the fine ones and the XY section at mid-height of every level
is read back (the reference driver's plotted output), and the run synchronises once.  The default FP32 plain
run also measures the metric's second form on the same case and step counts --
`forms.f16_mlp`: FP16 f - w storage with the learned closure, its network run on every
`--sgs-interval`-th update (default 4) and each cell's kept nu_t in between -- with its
roofline, its speed-up over the plain form and its long-run drag error against the plain
form (from the committed precision record; `--no-forms` skips it).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "D3Q27 MLUPS & % HBM roofline: FP32 plain vs FP16-store+learned SGS, same err"
BYTES_PER_UPDATE = {"f32": 216, "f16": 108, "bf16": 108}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="native", choices=["native", "reference"])
    p.add_argument("--config", type=int, default=2, choices=[1, 2])
    p.add_argument("--scale", type=float, default=1.0,
                   help="linear scale of the config-2 geometry (0.5: a 256x128x128 case for ncu captures)")
    p.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    p.add_argument("--form", default="single", choices=["single", "batch"])
    p.add_argument("--sgs", default="smagorinsky", choices=["smagorinsky", "mlp"],
                   help="mlp: the learned closure trained on decaying turbulence (packaged weights)")
    p.add_argument("--sgs-interval", type=int, default=4,
                   help="the learned closure's network on every K-th update, the kept nu_t in between "
                        "(16-bit storage; psl_set_sgs_mlp_interval; 1: every update)")
    p.add_argument("--batch-cases", type=int, default=64)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-sample-steps", type=int, default=2)
    p.add_argument("--no-forms", dest="forms", action="store_false",
                   help="only the selected form (default: FP32 plain also measures FP16 + learned closure)")
    return p.parse_args()


def workload(args):
    from periodicshiftlbm_b200.cases import config1, config2

    return config2(scale=args.scale) if args.config == 2 else config1()


def full_size_name() -> str:
    """The workload the committed ncu traffic figures were captured on (config 2, scale 1)."""
    from periodicshiftlbm_b200.cases import config2

    return config2().name


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(x: float, world: int) -> float:
    """The largest x over the ranks of the process group (x itself on one rank): the job's
    time is its slowest rank's.  Runs on the group's own device (CUDA for NCCL, host for gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank_step: float, steps: int, world: int, ms: float) -> float:
    """Whole-job throughput in millions of units per second: every rank (an independent
    replica) processes `units_per_rank_step` units per step, in the slowest rank's `ms`."""
    return units_per_rank_step * steps * world / (ms * 1e-3) / 1e6


# ------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons through NVML every
    `period_s` in a background thread while the timed region runs (read-only queries)."""

    REASONS = {
        "hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
        "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
        "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
        "sw_power_cap": "nvmlClocksEventReasonSwPowerCap",
        "hw_power_brake_slowdown": "nvmlClocksEventReasonHwPowerBrakeSlowdown",
    }

    def __init__(self, gpu_index: int, period_s: float = 0.005):
        self.gpu = gpu_index
        self.period = period_s
        self.samples = []
        self.thread = None

    def start(self):
        import threading

        try:
            import pynvml

            pynvml.nvmlInit()
            visible = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(visible.split(",")[self.gpu]) if visible else self.gpu
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nvml = None
            return
        self.stop_flag = threading.Event()

        def loop():
            nv = self.nvml
            while not self.stop_flag.is_set():
                try:
                    mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                    reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    self.samples.append((mhz, reasons))
                except Exception:
                    pass
                self.stop_flag.wait(self.period)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        if not self.thread:
            return None
        self.stop_flag.set()
        self.thread.join(timeout=2)
        if not self.samples:
            return None
        nv = self.nvml
        mhz = [m for m, _ in self.samples]
        active = sorted({name for name, attr in self.REASONS.items()
                         for _, r in self.samples if hasattr(nv, attr) and r & getattr(nv, attr)})
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": self.max_mhz, "reasons": active,
                "samples": len(self.samples), "source": "nvml"}


# ------------------------------------------------------------------------------------------
# measured peaks and the ncu traffic summary
# ------------------------------------------------------------------------------------------
def hbm_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def update_kernel(storage: str, sgs: str) -> str:
    """The coarse-grid update kernel the library launches for this form."""
    if sgs == "mlp":
        return "step_learned_warp_kernel"
    return "step_kernel_g" if storage in ("f16", "bf16") else "step_kernel"


def closure_interval(storage: str, sgs: str, interval: int) -> int:
    """Updates per run of the closure's network (1 unless a 16-bit form runs it on every
    interval-th update)."""
    return interval if sgs == "mlp" and storage in ("f16", "bf16") and interval > 1 else 1


def batch_traffic(storage: str, cells: int):
    """DRAM bytes per launch of the batched update: the per-cell traffic of the committed
    16-case capture (profiles/batch_step_kernel_batch16.md, FP32) times the cells."""
    path = os.path.join(REPO, "profiles", "batch_step_kernel_batch16.md")
    if storage != "f32" or not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_cell:\s*([0-9.eE+]+)", open(path).read())
    return round(float(m.group(1)) * cells) if m else None


def long_run_drag_error(interval: int = 1):
    """|C_d(FP16 + closure) / C_d(plain FP32) - 1| of the long-run means in the committed
    precision record (python -m periodicshiftlbm_b200.precision, 100,000 steps) for the
    closure run on every `interval`-th update, or None."""
    path = os.path.join(REPO, "periodicshiftlbm_b200", "data", "study_precision_sphere256.json")
    try:
        forms = json.load(open(path))["forms"]
        key = "f16+mlp" if interval <= 1 else f"f16+mlp{interval}"
        return round(abs(forms[key]["cd_mean"] / forms["f32"]["cd_mean"] - 1.0), 5)
    except (OSError, KeyError, ValueError):
        return None


def ncu_traffic(kernel: str, storage: str):
    """DRAM bytes read + written by one coarse-grid launch of `kernel`, from the committed
    ncu summary profiles/<kernel>_<storage>_sphere512.md (a full-size capture), or None."""
    path = os.path.join(REPO, "profiles", f"{kernel}_{storage}_sphere512.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


# ------------------------------------------------------------------------------------------
# native (CUDA) arm
# ------------------------------------------------------------------------------------------
def measure_form(args, cfg, storage: str, sgs: str, world: int, local: int, with_e2e: bool) -> dict:
    """One form of the update on config `cfg`: W warm-up steps, K device-timed steps (CUDA
    events on the grids' stream, max over ranks), the drag after those W + K steps, and
    (with_e2e) K more steps end to end through the public API with host buffers."""
    import torch

    from periodicshiftlbm_b200 import (
        applyCoarseFineGridCommunication,
        applyLocalCellUpdate,
        applyStreaming,
        getSphereForce,
        getSphereForceAsync,
        updateGrid,
    )
    from periodicshiftlbm_b200.cases import make_sphere_grids

    stream = torch.cuda.Stream()
    grids, case = make_sphere_grids(cfg, storage=storage)
    for g in grids:
        g.set_stream(stream.cuda_stream)
    if sgs == "mlp":
        from periodicshiftlbm_b200.sgs import load_params, set_sgs_mlp

        closure = load_params()
        for g in grids:
            set_sgs_mlp(g, closure, g.Info.res / grids[0].Info.res,
                        interval=args.sgs_interval if storage in ("f16", "bf16") else None)
    torch.cuda.synchronize()
    levels = len(grids)
    ev = {"coarse": [], "fine": []}

    def update(level, record):
        """updateGrid (flowAroundSphereMainSingle.cu:158-167) with events around the
        update launches when `record`."""
        g = grids[level]
        applyStreaming(g)
        if record:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            applyLocalCellUpdate(g)
            b.record(stream)
            ev["coarse" if level == 0 else "fine"].append((a, b))
        else:
            applyLocalCellUpdate(g)
        if level < levels - 1:
            update(level + 1, record)
            update(level + 1, record)
            applyCoarseFineGridCommunication(g, grids[level + 1])

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    # the timed steps: updateGrid, one library call per coarse step (psl_update_grid, which
    # updates the coarse cells away from the refinement block on a side stream beside the fine
    # updates and the transfer)
    for _ in range(args.warmup):
        updateGrid(grids, 0)
    torch.cuda.synchronize()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        updateGrid(grids, 0)
    t1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    ms = max_over_ranks(t0.elapsed_time(t1), world)
    # the update kernels' own launch times: CUDA events around each update launch in a few
    # serial steps right after the timed ones (one launch at a time on the grids' stream)
    for _ in range(min(args.steps, 8)):
        update(0, True)
    torch.cuda.synchronize()
    updates = cfg.updates_per_step()
    drag_after = float(getSphereForce(grids[-1], case)[0])
    out = {
        "storage": storage, "sgs": sgs, "updates": updates, "ms": ms, "levels": levels, "clocks": clocks,
        "value": job_rate(updates, args.steps, world, ms), "drag_after_timed": drag_after,
        "coarse_ms": statistics.mean(a.elapsed_time(b) for a, b in ev["coarse"]),
        "fine_ms": statistics.mean(a.elapsed_time(b) for a, b in ev["fine"]) if ev["fine"] else None,
    }
    # roofline of the dominant kernel: the coarse-grid update
    info0 = cfg.infos()[0]
    coarse_updates = info0.cellCount
    if cfg.refine:
        (i0, j0, k0), (i1, j1, k1) = cfg.refine
        coarse_updates -= (i1 - i0 - 4) * (j1 - j0 - 4) * (k1 - k0 - 4)
    every = closure_interval(storage, sgs, args.sgs_interval)
    # with a closure interval each update also moves the cell's kept nu_t (2 bytes): written
    # by the closure's run, read by the updates between
    bpu = BYTES_PER_UPDATE[storage] + (2 if every > 1 else 0)
    peak, peak_kind = hbm_peak()
    achieved = bpu * coarse_updates / (out["coarse_ms"] * 1e-3) / 1e9
    kernel = update_kernel(storage, sgs)
    label = kernel + " (coarse grid)"
    traffic = ncu_traffic(kernel, storage) if cfg.name == full_size_name() else None
    if every > 1:
        label = (f"{kernel} on every {every}th update, step_kernel_g with the kept nu_t between "
                 "(coarse grid, mean launch)")
        held = ncu_traffic("step_kernel_g_nu", storage) if cfg.name == full_size_name() else None
        # the network's run was captured at interval 1: add the nu_t it stores (2 bytes a cell)
        traffic = (round((traffic + 2 * coarse_updates + (every - 1) * held) / every)
                   if traffic and held else None)
    out["roofline"] = {
        "bound": "hbm", "kernel": label, "achieved": round(achieved, 1), "peak": peak,
        "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
        "traffic": traffic,
        "algorithmic_bytes_per_launch": bpu * coarse_updates,
        "launch_ms": round(out["coarse_ms"], 4),
        "fine_launch_ms": round(out["fine_ms"], 4) if out["fine_ms"] else None,
        "whole_step_frac": round(bpu * updates / (ms / args.steps * 1e-3) / 1e9 / peak, 4),
    }
    if with_e2e:
        # ---- end to end through the public API with host buffers ----
        from periodicshiftlbm_b200 import fillCoarseGridFromFine, sectionCut

        pinned_in = [torch.empty((27, g.cellCount), dtype=torch.float32).pin_memory() for g in grids]
        for g, h in zip(grids, pinned_in):
            g.read_populations(h.numpy())
        # every step's drag is copied to a pinned host array in stream order (no host wait
        # per step; the run synchronises once at the end)
        drag_hist = torch.zeros((max(1, args.steps), 3), dtype=torch.float64).pin_memory()
        # one untimed pass through the leg's other calls: a kernel's first launch in a process
        # loads it (tens to hundreds of ms); the upload below overwrites what the pass changed
        getSphereForceAsync(grids[-1], case, drag_hist.data_ptr())
        for lvl in range(levels - 2, -1, -1):
            fillCoarseGridFromFine(grids[lvl], grids[lvl + 1])
        for g in grids:
            sectionCut(g, "XY", g.Info.cellCountZ // 2)
        torch.cuda.synchronize()
        barrier()
        e0 = time.perf_counter()
        for g, h in zip(grids, pinned_in):
            g.write_populations(h.numpy())
        for s in range(args.steps):
            updateGrid(grids, 0)
            getSphereForceAsync(grids[-1], case, drag_hist.data_ptr() + s * 24)
        # the reference driver's output (flowAroundSphereMainSingle.cu:266-277): the coarse
        # levels filled from the fine ones, then the XY section at mid-height of every level
        for lvl in range(levels - 2, -1, -1):
            fillCoarseGridFromFine(grids[lvl], grids[lvl + 1])
        sections = [sectionCut(g, "XY", g.Info.cellCountZ // 2) for g in grids]
        torch.cuda.synchronize()
        drags = [float(v) for v in drag_hist[: args.steps, 0]]
        e_s = max_over_ranks(time.perf_counter() - e0, world)
        state_bytes = sum(h.numpy().nbytes for h in pinned_in)
        section_bytes = sum(sec.nbytes for sec in sections)
        out["e2e"] = {
            "value": round(job_rate(updates, args.steps, world, e_s * 1e3), 1),
            "unit": "MLUPS",
            "h2d_bytes_per_step": round(state_bytes / args.steps),
            "d2h_bytes_per_step": round(section_bytes / args.steps) + 24,
            "note": "the initial state uploaded from pinned host memory once per run; every step's FP64 "
                    "drag copied back to pinned host memory in stream order; at the end the coarse levels "
                    "filled from the fine ones and the XY section at mid-height of every level read back "
                    "(the reference driver's per-step drag and plotted sections, "
                    "flowAroundSphereMainSingle.cu:245-277); one synchronisation at the end",
        }
        out["drag_last"] = drags[-1] if drags else None
    for g in grids:
        g.close()
    torch.cuda.synchronize()
    return out


def run_native(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cfg = workload(args)
    main = measure_form(args, cfg, args.storage, args.sgs, world, local, with_e2e=True)
    levels = main["levels"]
    line = {
        "metric": METRIC,
        "value": round(main["value"], 1),
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(main["ms"] / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if args.storage == "f32" else f"{args.storage}-storage/f32-math",
        "data": "synthetic",
        "config": config_dict(cfg, args.storage, args.sgs, world, args.sgs_interval),
        "roofline": main["roofline"],
        "e2e": main["e2e"],
        # per coarse step on two levels: the coarse update as two launches (near slab, far
        # layers), two fine updates, the transfer as two launches (restriction, prolongation)
        "gpu_launches": args.steps * (6 if levels == 2 else 1 + 3 * (levels - 1)),
        "clocks": main["clocks"],
        "drag_after_timed": main["drag_after_timed"],
        "drag_last": main.get("drag_last"),
    }
    if args.forms and args.storage == "f32" and args.sgs == "smagorinsky":
        # the metric's second form on the same case and step counts: FP16 f - w storage +
        # the learned closure, against this FP32 plain run
        alt = measure_form(args, cfg, "f16", "mlp", world, local, with_e2e=False)
        plain_drag = main["drag_after_timed"]
        line["forms"] = {
            "f32_plain": {"value": round(main["value"], 1), "ms_per_step": round(main["ms"] / args.steps, 4),
                          "roofline_frac": main["roofline"]["frac"],
                          "whole_step_frac": main["roofline"]["whole_step_frac"],
                          "drag_after_timed": plain_drag},
            "f16_mlp": {"value": round(alt["value"], 1), "ms_per_step": round(alt["ms"] / args.steps, 4),
                        "speedup_vs_f32_plain": round(alt["value"] / main["value"], 3),
                        "closure_interval": args.sgs_interval,
                        "roofline": alt["roofline"], "clocks": alt["clocks"],
                        "drag_after_timed": alt["drag_after_timed"],
                        "drag_rel_vs_f32_plain": long_run_drag_error(args.sgs_interval),
                        "drag_rel_vs_f32_plain_after_timed": round(
                            abs(alt["drag_after_timed"] - plain_drag) / abs(plain_drag), 5),
                        "note": "drag_rel_vs_f32_plain: mean drag coefficient over steps 20,001-100,000 of the "
                                "half-scale case, FP16 + closure (the same interval) against plain FP32, "
                                "from the committed "
                                "precision record (periodicshiftlbm_b200/data/study_precision_sphere256.json); "
                                "..._after_timed: instantaneous drag after this run's warm-up + timed steps "
                                "from the same start, inside the start-up transient"},
        }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, args.cpu_sample_steps)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def config_dict(cfg, storage: str, sgs: str, world: int, interval: int = 1) -> dict:
    """The `config` of a bench line; the reference arm reports the same keys."""
    every = "" if interval <= 1 or storage == "f32" else f", network on every {interval}th update, kept nu_t between"
    return {
        "workload": cfg.name,
        "grid": [cfg.nx, cfg.ny, cfg.nz],
        "refine_block": cfg.refine,
        "storage": storage,
        "updates_per_step": cfg.updates_per_step(),
        "reference_formula_updates_per_step": cfg.reference_updates_per_step(),
        "collision": (f"cumulant + learned MLP closure (per-warp tensor-core MMAs{every})" if sgs == "mlp" else
                      "cumulant + Smagorinsky" if cfg.smagorinsky else "cumulant"),
        "l2": "inputs larger than L2 (no flush)" if cfg.refine else "state fits partly in L2",
        "parallelism": f"replicas x{world}",
    }


# ------------------------------------------------------------------------------------------
# the reference's own CPU code (oracle/_ref, compiled for the host): CPU baseline / arm
# ------------------------------------------------------------------------------------------
def _ref_case(cfg):
    from oracle.bindings import SphereCase as RefCase

    return RefCase(nx=cfg.nx, ny=cfg.ny, nz=cfg.nz, sphere=tuple(cfg.sphere), radius=cfg.radius, u_in=cfg.u_in,
                   nu=cfg.nu, smagorinsky=cfg.smagorinsky, wall_mode=cfg.wall_mode, seed=cfg.seed, noise=cfg.noise,
                   refine=cfg.refine)


def _ref_lib():
    from oracle.bindings import RefLib, ref_available

    if ref_available():
        return RefLib(), "reference"
    from oracle.bindings import OracleLib

    return OracleLib(), "port"


def cpu_baseline(cfg, sample_steps):
    lib, kind = _ref_lib()
    sim = lib.sim(_ref_case(cfg))
    t = time.perf_counter()
    sim.run(sample_steps)
    dt = time.perf_counter() - t
    value = cfg.updates_per_step() * sample_steps / dt / 1e6
    sim.close()
    return {"value": round(value, 2), "unit": "MLUPS", "cores": os.cpu_count(), "kind": kind,
            "sample": f"{sample_steps} coarse steps of {cfg.name} ({cfg.updates_per_step() * sample_steps} updates, "
                      f"{dt:.1f} s), g++ -O3 -fopenmp, OMP threads = {os.environ.get('OMP_NUM_THREADS', os.cpu_count())}"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cfg = workload(args)
    lib, kind = _ref_lib()
    sim = lib.sim(_ref_case(cfg))
    budget_s = 150.0
    for _ in range(min(args.warmup, 1)):
        sim.run(1)
    t0 = time.perf_counter()
    done = 0
    while done < args.steps:
        sim.run(1)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    value = cfg.updates_per_step() * done / dt / 1e6
    sample = (f"{done} of {args.steps} coarse steps of {cfg.name} (time-capped at {budget_s:.0f} s), "
              f"warm-up {min(args.warmup, 1)} step")
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": world, "steps": done,
        "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / max(done, 1), 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": config_dict(cfg, "f32", "smagorinsky", world),
        "cpu_baseline": {"value": round(value, 2), "unit": "MLUPS", "cores": os.cpu_count(), "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    sim.close()
    print(json.dumps(line), flush=True)


def run_batch(args):
    """The batched form on one GPU (replicas on more)."""
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from periodicshiftlbm_b200 import getSphereForce
    from periodicshiftlbm_b200.batch import Batch, batch_configs, make_batch_grids

    cfgs = batch_configs(args.batch_cases)
    grids, cases = make_batch_grids(cfgs, storage=args.storage)
    b = Batch(grids)
    tuning = b.autotune(3)
    stream = torch.cuda.ExternalStream(b.stream)
    cells = b.cells()
    b.run(args.warmup)
    b.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    b.run(args.steps)
    t1.record(stream)
    b.synchronize()
    clocks = sampler.stop()
    ms = max_over_ranks(t0.elapsed_time(t1), world)
    value = job_rate(cells, args.steps, world, ms)
    bpu = BYTES_PER_UPDATE[args.storage]
    peak, peak_kind = hbm_peak()
    achieved = bpu * cells / (ms / args.steps * 1e-3) / 1e9

    # end to end: states from pinned host memory, K graph replays, per-case drag and the
    # final states back to the host
    pinned = [torch.empty((27, g.cellCount), dtype=torch.float32).pin_memory() for g in grids]
    for g, h in zip(grids, pinned):
        g.read_populations(h.numpy())
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    for g, h in zip(grids, pinned):
        g.write_populations(h.numpy())
    b.run(args.steps)
    drags = [float(getSphereForce(g, c)[0]) for g, c in zip(grids, cases)]
    for g, h in zip(grids, pinned):
        g.read_populations(h.numpy())
    e_s = max_over_ranks(time.perf_counter() - e0, world)
    state_bytes = sum(h.numpy().nbytes for h in pinned)
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.storage == "f32" else f"{args.storage}-storage/f32-math", "data": "synthetic",
        "config": {"workload": f"batch{len(cfgs)}_sphere_x64-192_re1e2-1e6", "cases": len(cfgs), "cells": cells,
                   "storage": args.storage, "tuning": tuning, "graph": "one step per replay",
                   "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": "batch_step_kernel", "achieved": round(achieved, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": batch_traffic(args.storage, cells),
                     "algorithmic_bytes_per_launch": bpu * cells},
        "e2e": {"value": round(job_rate(cells, args.steps, world, e_s * 1e3), 1), "unit": "MLUPS",
                "h2d_bytes_per_step": round(state_bytes / args.steps),
                "d2h_bytes_per_step": round(state_bytes / args.steps) + 24 * len(cfgs) // max(args.steps, 1),
                "note": "states uploaded once and downloaded once per run, per-case drag read at the end"},
        "gpu_launches": 3 * args.steps,
        "clocks": clocks,
    }
    b.close()
    for g in grids:
        g.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.form == "batch":
        run_batch(args)
    else:
        run_native(args)


if __name__ == "__main__":
    main()
