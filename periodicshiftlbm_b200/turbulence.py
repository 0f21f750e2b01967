"""Decaying homogeneous turbulence in a periodic box, and the training / evaluation of the
learned subgrid closure on it.

Box.  M physical cells per axis on a grid of (M+1) x (M+1) x M cells: x and y are made
periodic by applyBCPeriodicX/Y after streaming (periodicXY.h:11-101), whose copies make the
first and last layer the same physical cell; z is periodic through the periodic-shift
addressing itself.  All cells are fluid.

Start.  A seeded random-phase, divergence-free velocity field with
E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4, scaled to u_rms = 0.04 (per component), rho = 1,
populations at equilibrium.  The fine box (2M) and the coarse box (M) start from the same
band-limited field (the coarse one samples every second fine cell; the spectrum has no
energy near the coarse Nyquist wavenumber).

Closure study (``study``): fine plain-solver runs (Smagorinsky C_s = 0.1, FP32) from
several seeds are box-filtered 2x into training samples (psl_sgs_trainer_add_filtered),
the MLP is trained with the library's CUDA kernels, and coarse runs with Smagorinsky and
with the closure are compared on the energy spectrum against the box-filtered fine run of
a held-out seed.  Under acoustic scaling one coarse step is two fine steps and the fine
lattice viscosity is twice the coarse one.
"""
from __future__ import annotations

import json
import time

import numpy as np

from .grid import (
    GridStruct,
    InfoStruct,
    applyBCPeriodicX,
    applyBCPeriodicY,
    applyLocalCellUpdate,
    applyStreaming,
    setSmagorinskyConstant,
)
from ._lib import call
from .sgs import Trainer, init_params, mlp_infer, set_sgs_mlp, smagorinsky_nu_t


def box_grid(M: int, nu: float, storage: str = "f32", cs: float = 0.0) -> GridStruct:
    g = GridStruct(InfoStruct(cellCountX=M + 1, cellCountY=M + 1, cellCountZ=M, nu=nu), storage=storage)
    setSmagorinskyConstant(g, cs)
    return g


def initial_velocity(M: int, seed: int, u_rms: float = 0.04, k0: float = 4.0) -> np.ndarray:
    """[3, z, y, x] float32 velocity on an M^3 periodic lattice (component 0 along x)."""
    try:
        from scipy import fft as sfft

        irfftn = lambda a: sfft.irfftn(a, s=(M, M, M), axes=(1, 2, 3), workers=-1)  # noqa: E731
    except ImportError:  # pragma: no cover
        irfftn = lambda a: np.fft.irfftn(a, s=(M, M, M), axes=(1, 2, 3))  # noqa: E731
    rng = np.random.default_rng(seed)
    shape = (M, M, M // 2 + 1)
    kz = np.fft.fftfreq(M, 1.0 / M).astype(np.float32)[:, None, None]
    ky = np.fft.fftfreq(M, 1.0 / M).astype(np.float32)[None, :, None]
    kx = np.fft.rfftfreq(M, 1.0 / M).astype(np.float32)[None, None, :]
    a = np.empty((3,) + shape, dtype=np.complex64)
    for c in range(3):
        a[c].real = rng.standard_normal(shape, dtype=np.float32)
        a[c].imag = rng.standard_normal(shape, dtype=np.float32)
    k2 = kx * kx + ky * ky + kz * kz
    safe = np.where(k2 > 0, k2, 1.0).astype(np.float32)
    proj = (a[0] * kx + a[1] * ky + a[2] * kz) / safe
    a[0] -= kx * proj  # divergence-free: k . a = 0
    a[1] -= ky * proj
    a[2] -= kz * proj
    del proj
    k = np.sqrt(k2)
    amp = np.where(k2 > 0, np.sqrt(k2 * k2 * np.exp(-2.0 * (k / k0) ** 2) / (4.0 * np.pi * safe)), 0.0).astype(np.float32)
    norm = np.sqrt((np.abs(a) ** 2).sum(0))
    a *= np.where(norm > 0, amp / np.maximum(norm, 1e-30), 0.0).astype(np.float32)[None]
    del norm, amp, k
    u = irfftn(a).astype(np.float64)
    u *= u_rms / np.sqrt(np.mean(u ** 2))
    return u.astype(np.float32)


def fill_from_velocity(grid: GridStruct, u: np.ndarray):
    """feq(rho = 1, u) on the (M+1) x (M+1) x M box (duplicated x/y layers copied)."""
    M = u.shape[-1]
    N = (M + 1) * (M + 1) * M
    ix = np.arange(M + 1) % M
    rho_u = np.empty((4, M, M + 1, M + 1), dtype=np.float32)
    rho_u[0] = 1.0
    for c in range(3):
        rho_u[1 + c] = u[c][:, ix][:, :, ix]
    rho_u = np.ascontiguousarray(rho_u.reshape(4, N))
    call("psl_fill_equilibrium_field", grid.handle, rho_u.ctypes.data)


def step(grid: GridStruct):
    """One step of the periodic box: streaming, the x and y periodic copies, the update."""
    applyStreaming(grid)
    applyBCPeriodicX(grid)
    applyBCPeriodicY(grid)
    applyLocalCellUpdate(grid)


def velocity(grid: GridStruct) -> np.ndarray:
    """[3, z, y, x] velocity of the M^3 physical cells (FP64)."""
    M = grid.Info.cellCountZ
    m = grid.macroscopic().reshape(4, M, M + 1, M + 1)
    return np.ascontiguousarray(m[1:, :, :M, :M])


def box_filter(u: np.ndarray) -> np.ndarray:
    c, M = u.shape[0], u.shape[-1]
    return u.reshape(c, M // 2, 2, M // 2, 2, M // 2, 2).mean(axis=(2, 4, 6))


def energy_spectrum(u: np.ndarray):
    """Shell-summed kinetic energy E(k), k = 0 .. M/2 (integer shells of |k|)."""
    M = u.shape[-1]
    uh = np.fft.rfftn(u, axes=(1, 2, 3)) / M ** 3
    e = 0.5 * (np.abs(uh) ** 2).sum(0)
    w = np.full(M // 2 + 1, 2.0)
    w[0] = 1.0
    if M % 2 == 0:
        w[-1] = 1.0
    e = e * w[None, None, :]
    kz = np.fft.fftfreq(M, 1.0 / M)[:, None, None]
    ky = np.fft.fftfreq(M, 1.0 / M)[None, :, None]
    kx = np.fft.rfftfreq(M, 1.0 / M)[None, None, :]
    shell = np.rint(np.sqrt(kx * kx + ky * ky + kz * kz)).astype(int)
    E = np.bincount(shell.ravel(), weights=e.ravel(), minlength=M // 2 + 1)[: M // 2 + 1]
    return np.arange(M // 2 + 1), E


def spectrum_error(E: np.ndarray, E_ref: np.ndarray, kmax: int) -> float:
    """RMS over shells 1..kmax of log(E / E_ref)."""
    r = np.log(np.maximum(E[1:kmax + 1], 1e-300) / np.maximum(E_ref[1:kmax + 1], 1e-300))
    return float(np.sqrt(np.mean(r * r)))


def run(grid: GridStruct, steps: int) -> float:
    """Advance `steps` steps; returns the wall time in seconds (synchronised)."""
    grid.synchronize()
    t = time.perf_counter()
    for _ in range(steps):
        step(grid)
    grid.synchronize()
    return time.perf_counter() - t


COARSE_FORMS = (("smagorinsky_f32", "f32", False), ("smagorinsky_f16", "f16", False), ("closure_f16", "f16", True),
                ("closure_f32", "f32", True))


def evaluate_coarse(M: int, params: dict, u0_fine: np.ndarray, E_ref: np.ndarray, eval_steps: int, nu: float,
                    cs: float, forms=COARSE_FORMS, say=None) -> dict:
    """A-posteriori runs of the coarse box (M^3, every second cell of the fine start field
    `u0_fine`) with Smagorinsky and with the closure, each after `eval_steps` steps compared
    on the energy spectrum against `E_ref` (the box-filtered fine run)."""
    coarse_u0 = np.ascontiguousarray(u0_fine[:, ::2, ::2, ::2])
    kmax = M // 2
    results = {}
    for name, storage, closure in forms:
        g = box_grid(M, nu, storage=storage, cs=cs)
        if closure:
            set_sgs_mlp(g, params, 1.0)
        fill_from_velocity(g, coarse_u0)
        sec = run(g, eval_steps)
        health = g.health()
        _, E = energy_spectrum(velocity(g))
        results[name] = {"spectrum_error": spectrum_error(E, E_ref, kmax),
                         "spectrum_error_k_le_32": spectrum_error(E, E_ref, min(32, kmax)),
                         "mlups": g.cellCount * eval_steps / sec / 1e6, "health": health,
                         "energy": float(E.sum()), "E": E.tolist()}
        g.close()
        if say:
            say(f"{name}: {results[name]['spectrum_error']:.4f}")
    return results


def filtered_fine_spectrum(M: int, seed: int, eval_steps: int, nu: float, cs: float, k0: float = 4.0):
    """The held-out reference: a (2M)^3 fine run (viscosity 2 nu, Smagorinsky cs) of seed
    `seed` after 2 eval_steps steps, box-filtered 2x; returns (start field, E_ref, seconds)."""
    fine = box_grid(2 * M, 2 * nu, cs=cs)
    u0 = initial_velocity(2 * M, seed, k0=k0)
    fill_from_velocity(fine, u0)
    sec = run(fine, 2 * eval_steps)
    _, E_ref = energy_spectrum(box_filter(velocity(fine)))
    fine.close()
    return u0, E_ref, sec


def study(M: int = 256, seeds=(0, 1, 2, 3, 4, 5, 6, 7), eval_seed: int = 100, snapshots=(2000, 4000, 6000, 8000),
          eval_steps: int = 4000, nu: float = 1e-5, cs: float = 0.1, stride: int = 16, train_steps: int = 4000,
          batch: int = 65536, lr: float = 1e-3, log=None) -> dict:
    """Train the closure on box-filtered fine runs and evaluate it against Smagorinsky."""
    say = log or (lambda *a: None)
    per_snap = -(-M ** 3 // stride)
    trainer = Trainer(len(seeds) * len(snapshots) * per_snap)
    t0 = time.perf_counter()
    for s in seeds:
        fine = box_grid(2 * M, 2 * nu, cs=cs)
        fill_from_velocity(fine, initial_velocity(2 * M, s))
        done = 0
        for j, target in enumerate(snapshots):
            run(fine, target - done)
            done = target
            trainer.add_filtered(fine, M, stride, phase=(7 * s + j) % stride)
        say(f"seed {s}: {trainer.count} samples")
        fine.close()
    gen_s = time.perf_counter() - t0
    x, t = trainer.samples(0, min(trainer.count, 2_000_000))
    params = init_params(x, t, seed=0)
    trainer.params = params
    losses = []
    chunk = max(1, train_steps // 20)
    t1 = time.perf_counter()
    for _ in range(0, train_steps, chunk):
        losses.append(trainer.train(chunk, batch, lr, seed=len(losses) + 1))
    train_s = time.perf_counter() - t1
    params = trainer.params

    # held-out seed: a-priori error of the closure and of Smagorinsky on its filtered snapshot,
    # and the box-filtered fine spectrum after 2 * eval_steps fine steps
    fine = box_grid(2 * M, 2 * nu, cs=cs)
    u0 = initial_velocity(2 * M, eval_seed)
    fill_from_velocity(fine, u0)
    fine_s = run(fine, 2 * eval_steps)
    held = Trainer(per_snap)
    held.add_filtered(fine, M, stride, phase=3)
    hx, ht = held.samples()
    held.close()
    pred = mlp_infer(params, hx).astype(np.float64)
    smag = smagorinsky_nu_t(hx, nu, cs)
    apriori = {"mse_closure": float(np.mean((pred - ht) ** 2)), "mse_smagorinsky": float(np.mean((smag - ht) ** 2)),
               "mse_zero": float(np.mean(ht.astype(np.float64) ** 2)), "target_mean": float(np.mean(ht))}
    k, E_ref = energy_spectrum(box_filter(velocity(fine)))
    fine_mlups = fine.cellCount * 2 * eval_steps / fine_s / 1e6
    fine.close()
    results = evaluate_coarse(M, params, u0, E_ref, eval_steps, nu, cs, say=say)
    trainer.close()
    return {"M": M, "seeds": list(seeds), "eval_seed": eval_seed, "snapshots_fine_steps": list(snapshots),
            "eval_coarse_steps": eval_steps, "nu": nu, "cs": cs, "samples": int(len(seeds) * len(snapshots) * per_snap),
            "train_steps": train_steps, "batch": batch, "lr": lr, "loss_curve": losses, "generate_s": gen_s,
            "train_s": train_s, "fine_mlups": fine_mlups, "apriori": apriori, "runs": results,
            "E_ref": E_ref.tolist(), "E_ref_energy": float(E_ref.sum()), "params": {k2: np.asarray(v).tolist() for k2, v in params.items()}}


def main(argv=None):
    import argparse
    import sys

    ap = argparse.ArgumentParser(description="train and evaluate the learned closure on decaying turbulence")
    ap.add_argument("--M", type=int, default=256)
    ap.add_argument("--seeds", type=int, default=8)
    ap.add_argument("--snapshots", default="2000,4000,6000,8000")
    ap.add_argument("--eval-steps", type=int, default=4000)
    ap.add_argument("--stride", type=int, default=16)
    ap.add_argument("--train-steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    res = study(a.M, tuple(range(a.seeds)), snapshots=tuple(int(v) for v in a.snapshots.split(",")),
                eval_steps=a.eval_steps, stride=a.stride, train_steps=a.train_steps, batch=a.batch,
                log=lambda *m: print(*m, file=sys.stderr, flush=True))
    text = json.dumps({"command": "python -m periodicshiftlbm_b200.turbulence " + " ".join(argv or sys.argv[1:]), **res})
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(text)
    print(json.dumps({k: v for k, v in res.items() if k not in ("E_ref", "params")} | {
        "runs": {n: {kk: vv for kk, vv in r.items() if kk != "E"} for n, r in res["runs"].items()}}))


if __name__ == "__main__":
    main()
