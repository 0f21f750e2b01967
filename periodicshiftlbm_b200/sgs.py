"""The learned subgrid closure from Python: parameters as a dict of numpy arrays
(w1 [32,10], b1 [32], w2 [32,32], b2 [32], w3 [32], b3, in_shift [10], in_scale [10],
out_scale), attached to a grid (psl_set_sgs_mlp) or evaluated alone on the tensor cores
(psl_sgs_mlp_infer)."""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

from ._lib import PslSgsMlp, call

FIELDS = ("w1", "b1", "w2", "b2", "w3", "b3", "in_shift", "in_scale", "out_scale")


def to_c(p: dict) -> PslSgsMlp:
    m = PslSgsMlp()
    for name in FIELDS:
        v = np.asarray(p[name], dtype=np.float32)
        if v.ndim == 0:
            setattr(m, name, float(v))
        else:
            ctypes.memmove(ctypes.addressof(getattr(m, name)), np.ascontiguousarray(v).ctypes.data, v.nbytes)
    return m


def from_c(m: PslSgsMlp) -> dict:
    out = {}
    for name in FIELDS:
        v = getattr(m, name)
        out[name] = np.float32(v) if isinstance(v, float) else np.ctypeslib.as_array(v).astype(np.float32).copy()
    return out


def set_sgs_mlp(grid, p: dict | None, filter_width: float = 1.0, interval: int | None = None):
    """Use the closure in the grid's update kernel (None: back to Smagorinsky).  `interval`
    (psl_set_sgs_mlp_interval): run the network on every interval-th update only and relax
    with each cell's kept nu_t in between (FP16 / BF16 storage); None keeps the grid's
    setting (1 unless set)."""
    if p is None:
        call("psl_set_sgs_mlp", grid.handle, None, ctypes.c_float(filter_width))
    else:
        m = to_c(p)
        call("psl_set_sgs_mlp", grid.handle, ctypes.byref(m), ctypes.c_float(filter_width))
    if interval is not None:
        set_sgs_mlp_interval(grid, interval)


def set_sgs_mlp_interval(grid, interval: int):
    """psl_set_sgs_mlp_interval: the closure runs on every `interval`-th update of the grid."""
    call("psl_set_sgs_mlp_interval", grid.handle, int(interval))


def mlp_infer(p: dict, x: np.ndarray) -> np.ndarray:
    """nu_t of raw feature rows x [n, 10] through the tensor-core device code."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.shape[0], dtype=np.float32)
    m = to_c(p)
    call("psl_sgs_mlp_infer", ctypes.byref(m), x.ctypes.data, x.shape[0], out.ctypes.data)
    return out


class Trainer:
    """psl_sgs_trainer: training samples on the device, CUDA forward/backward kernels and
    Adam (include/psl.h)."""

    def __init__(self, capacity: int):
        self._h = ctypes.c_void_p()
        call("psl_sgs_trainer_create", ctypes.c_longlong(int(capacity)), ctypes.byref(self._h))

    def close(self):
        if self._h and self._h.value:
            from . import _lib

            _lib.lib().psl_sgs_trainer_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def count(self) -> int:
        n = ctypes.c_longlong()
        call("psl_sgs_trainer_count", self._h, ctypes.byref(n))
        return n.value

    def clear(self):
        call("psl_sgs_trainer_clear", self._h)

    def add_samples(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        call("psl_sgs_trainer_add_samples", self._h, x.ctypes.data, t.ctypes.data, ctypes.c_longlong(x.shape[0]))

    def add_filtered(self, fine_grid, M: int, stride: int = 1, phase: int = 0):
        call("psl_sgs_trainer_add_filtered", self._h, fine_grid.handle, int(M), int(stride), ctypes.c_uint(phase))

    def samples(self, first: int = 0, n: int | None = None):
        n = self.count - first if n is None else n
        x = np.empty((n, 10), dtype=np.float32)
        t = np.empty(n, dtype=np.float32)
        call("psl_sgs_trainer_get_samples", self._h, ctypes.c_longlong(first), ctypes.c_longlong(n), x.ctypes.data,
             t.ctypes.data)
        return x, t

    @property
    def params(self) -> dict:
        m = PslSgsMlp()
        call("psl_sgs_trainer_get_params", self._h, ctypes.byref(m))
        return from_c(m)

    @params.setter
    def params(self, p: dict):
        m = to_c(p)
        call("psl_sgs_trainer_set_params", self._h, ctypes.byref(m))

    def gradient(self, first: int, count: int):
        """(mean loss, gradient dict w1..b3) over samples [first, first + count)."""
        g = PslSgsMlp()
        loss = ctypes.c_double()
        call("psl_sgs_trainer_gradient", self._h, ctypes.c_longlong(first), ctypes.c_longlong(count), ctypes.byref(g),
             ctypes.byref(loss))
        d = from_c(g)
        return loss.value, {k: d[k] for k in ("w1", "b1", "w2", "b2", "w3", "b3")}

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 1) -> float:
        loss = ctypes.c_double()
        call("psl_sgs_trainer_train", self._h, int(steps), int(batch), ctypes.c_float(lr), ctypes.c_uint(seed),
             ctypes.byref(loss))
        return loss.value


def init_params(x: np.ndarray, t: np.ndarray, seed: int = 0) -> dict:
    """He-initialised weights with the normalisation taken from the samples: in_shift and
    in_scale standardise each feature (a constant feature keeps scale 1), out_scale is the
    mean target."""
    rng = np.random.default_rng(seed)
    x = np.asarray(x, dtype=np.float64)
    mean = x.mean(0)
    std = x.std(0)
    scale = np.where(std > 1e-12 * np.maximum(np.abs(mean), 1e-30), 1.0 / np.maximum(std, 1e-30), 1.0)
    return {
        "w1": rng.normal(0.0, np.sqrt(2.0 / 10), (32, 10)),
        "b1": np.zeros(32),
        "w2": rng.normal(0.0, np.sqrt(2.0 / 32), (32, 32)),
        "b2": np.zeros(32),
        "w3": rng.normal(0.0, np.sqrt(1.0 / 32), 32),
        "b3": np.float64(0.0),
        "in_shift": mean,
        "in_scale": scale,
        "out_scale": np.float64(max(float(np.mean(t)), 1e-12)),
    }


def smagorinsky_nu_t(x: np.ndarray, nu: float, cs: float) -> np.ndarray:
    """Eddy viscosity of the Smagorinsky rate (cellFunctions.h:157-198) from the same
    features: tau_LES = tau/2 + sqrt(tau^2 + 18 C_s |Pi|)/2 with |Pi| = x[:, 7] (per unit
    density), nu_t = (tau_LES - 1/2)/3 - nu."""
    tau = 3.0 * nu + 0.5
    tau_les = 0.5 * tau + 0.5 * np.sqrt(tau * tau + 18.0 * cs * np.asarray(x, dtype=np.float64)[:, 7])
    return (tau_les - 0.5) / 3.0 - nu


PACKAGED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "closure_turbulence256.json")


def load_params(path: str = PACKAGED) -> dict:
    """Closure parameters saved by ``save_params`` (the packaged file holds the closure
    trained on the 512^3 -> 256^3 decaying-turbulence runs)."""
    with open(path) as fh:
        d = json.load(fh)
    return {k: np.asarray(d[k], dtype=np.float64) for k in FIELDS}


def save_params(p: dict, path: str, **meta):
    d = {k: np.asarray(p[k], dtype=np.float64).tolist() for k in FIELDS}
    d.update(meta)
    with open(path, "w") as fh:
        json.dump(d, fh)
