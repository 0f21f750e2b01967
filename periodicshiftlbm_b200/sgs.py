"""The learned subgrid closure from Python: parameters as a dict of numpy arrays
(w1 [32,10], b1 [32], w2 [32,32], b2 [32], w3 [32], b3, in_shift [10], in_scale [10],
out_scale), attached to a grid (psl_set_sgs_mlp) or evaluated alone on the tensor cores
(psl_sgs_mlp_infer)."""
from __future__ import annotations

import ctypes

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


def set_sgs_mlp(grid, p: dict | None, filter_width: float = 1.0):
    """Use the closure in the grid's update kernel (None: back to Smagorinsky)."""
    if p is None:
        call("psl_set_sgs_mlp", grid.handle, None, ctypes.c_float(filter_width))
    else:
        m = to_c(p)
        call("psl_set_sgs_mlp", grid.handle, ctypes.byref(m), ctypes.c_float(filter_width))


def mlp_infer(p: dict, x: np.ndarray) -> np.ndarray:
    """nu_t of raw feature rows x [n, 10] through the tensor-core device code."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.shape[0], dtype=np.float32)
    m = to_c(p)
    call("psl_sgs_mlp_infer", ctypes.byref(m), x.ctypes.data, x.shape[0], out.ctypes.data)
    return out
