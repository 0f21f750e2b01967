"""CPU oracle of the learned subgrid closure: features, forward pass and loss gradients.

ORACLE / TEST INFRASTRUCTURE ONLY -- the checker, never the thing measured or shipped.
The closure has no counterpart in the reference; this file restates the library's own
definition (include/psl.h, psl_sgs_mlp) in numpy:

    x  = 10 features of a cell (6 components of Pi = (C - rho/3 I)/rho from the
         second-order central moments, tr Pi, |Pi|, det Pi / |Pi|^2, filter width)
    x' = (x - in_shift) * in_scale
    h1 = relu(W1 x' + b1), h2 = relu(W2 h1 + b2)
    nu_t = out_scale * softplus(w3 . h2 + b3)

`forward_device` mirrors the tensor-core evaluation (FP16 weights, FP16 inputs and hidden
activations, FP32 accumulation); `forward64` / `loss_and_grad64` are the exact FP64
reference the training kernels' gradients are checked against (mean squared error on
nu_t / out_scale).
"""
from __future__ import annotations

import numpy as np

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1])
CZ = np.array([0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1])

PARAM_SHAPES = {"w1": (32, 10), "b1": (32,), "w2": (32, 32), "b2": (32,), "w3": (32,), "b3": ()}


def features(f: np.ndarray, width: float) -> np.ndarray:
    """f: [27, n] populations -> [n, 10] features (FP64)."""
    f = np.asarray(f, dtype=np.float64)
    rho = f.sum(0)
    ux = (CX[:, None] * f).sum(0) / rho
    uy = (CY[:, None] * f).sum(0) / rho
    uz = (CZ[:, None] * f).sum(0) / rho
    dx = CX[:, None] - ux[None]
    dy = CY[:, None] - uy[None]
    dz = CZ[:, None] - uz[None]

    def cm(a, b):
        return (a * b * f).sum(0)

    third = rho / 3.0
    pxx = (cm(dx, dx) - third) / rho
    pyy = (cm(dy, dy) - third) / rho
    pzz = (cm(dz, dz) - third) / rho
    pxy = cm(dx, dy) / rho
    pxz = cm(dx, dz) / rho
    pyz = cm(dy, dz) / rho
    n2 = pxx ** 2 + pyy ** 2 + pzz ** 2 + 2 * (pxy ** 2 + pxz ** 2 + pyz ** 2)
    det = pxx * (pyy * pzz - pyz * pyz) - pxy * (pxy * pzz - pyz * pxz) + pxz * (pxy * pyz - pyy * pxz)
    return np.stack([pxx, pyy, pzz, pxy, pxz, pyz, pxx + pyy + pzz, np.sqrt(n2), det / (n2 + 1e-30),
                     np.full_like(rho, width)], axis=1)


def softplus(z):
    return np.where(z > 20.0, z, np.log1p(np.exp(np.minimum(z, 20.0))))


def forward_device(p: dict, x: np.ndarray) -> np.ndarray:
    """nu_t as the tensor-core paths compute it: normalised features x * scale + offset
    (offset = -shift * scale, FP32), FP16 operands, the layer-1 biases as FP16 weights of a
    constant input 1, FP32 accumulation, ReLU, FP16 activations, FP32 layer-2 biases."""
    h16 = np.float16
    scale = p["in_scale"].astype(np.float32)
    offset = (-p["in_shift"] * p["in_scale"]).astype(np.float32)
    xn = (x.astype(np.float64) * scale + offset).astype(np.float32).astype(h16)
    w1 = p["w1"].astype(h16).astype(np.float32)
    w2 = p["w2"].astype(h16).astype(np.float32)
    w3 = p["w3"].astype(h16).astype(np.float32)
    a1 = xn.astype(np.float32) @ w1.T + p["b1"].astype(h16).astype(np.float32)
    h1 = np.maximum(a1, 0).astype(h16).astype(np.float32)
    a2 = h1 @ w2.T
    h2 = np.maximum(a2 + p["b2"].astype(np.float32), 0).astype(h16).astype(np.float32)
    z = h2 @ w3 + np.float32(p["b3"])
    return (np.float32(p["out_scale"]) * softplus(z.astype(np.float64))).astype(np.float32)


def forward64(p: dict, x: np.ndarray):
    xn = (x - p["in_shift"]) * p["in_scale"]
    a1 = xn @ p["w1"].T + p["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ p["w2"].T + p["b2"]
    h2 = np.maximum(a2, 0)
    z = h2 @ p["w3"] + p["b3"]
    return xn, a1, h1, a2, h2, z


def loss_and_grad64(p: dict, x: np.ndarray, target: np.ndarray):
    """Mean over samples of (softplus(z) - target / out_scale)^2 and its gradient with
    respect to w1, b1, w2, b2, w3, b3 (FP64)."""
    p = {k: np.asarray(v, dtype=np.float64) for k, v in p.items()}
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64) / p["out_scale"]
    xn, a1, h1, a2, h2, z = forward64(p, x)
    y = softplus(z)
    n = x.shape[0]
    r = y - t
    loss = float(np.mean(r * r))
    dy = 2.0 * r / n
    dz = dy / (1.0 + np.exp(-np.minimum(z, 50.0)))  # softplus' = sigmoid
    g = {"w3": h2.T @ dz, "b3": np.array(dz.sum())}
    dh2 = np.outer(dz, p["w3"]) * (a2 > 0)
    g["w2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ p["w2"]) * (a1 > 0)
    g["w1"] = dh1.T @ xn
    g["b1"] = dh1.sum(0)
    return loss, g


def random_params(seed: int, scale: float = 0.3) -> dict:
    rng = np.random.default_rng(seed)
    p = {k: rng.normal(0.0, scale, s) for k, s in PARAM_SHAPES.items()}
    p["b3"] = np.float64(rng.normal(0.0, scale))
    p["in_shift"] = rng.normal(0.0, 1e-3, 10)
    p["in_shift"][9] = 1.0  # the width feature is 1 on a uniform grid
    p["in_scale"] = np.abs(rng.normal(300.0, 50.0, 10))
    p["out_scale"] = np.float64(0.01)
    return p


def filtered_samples(fine_f: np.ndarray, M: int, rescale_f2c) -> tuple:
    """Training samples of a fine periodic box as the library's filter defines them.

    fine_f: logical-order populations [27, N] of the (2M+1) x (2M+1) x 2M fine box;
    rescale_f2c(f27) -> f27: the fine-to-coarse moment rescaling.  Returns (features
    [M^3, 10], targets [M^3]) for coarse cells in row-major order (x fastest)."""
    F = 2 * M
    f = np.asarray(fine_f, dtype=np.float64).reshape(27, F, F + 1, F + 1)[:, :, :F, :F]  # [q, z, y, x]
    rho = f.sum(0)
    u = np.stack([(CX[:, None, None, None] * f).sum(0), (CY[:, None, None, None] * f).sum(0),
                  (CZ[:, None, None, None] * f).sum(0)]) / rho

    def filt(a):
        return a.reshape(a.shape[:-3] + (M, 2, M, 2, M, 2)).mean(axis=(-5, -3, -1))

    fbar = filt(f).reshape(27, -1)
    fc = np.stack([rescale_f2c(fbar[:, i].astype(np.float32)) for i in range(fbar.shape[1])], axis=1)
    x = features(fc, 1.0)
    ub = np.stack([(CX[:, None] * fc).sum(0), (CY[:, None] * fc).sum(0), (CZ[:, None] * fc).sum(0)]) / fc.sum(0)
    ub = ub.reshape(3, M, M, M)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    tau = {ab: filt(u[ab[0]] * u[ab[1]]) - ub[ab[0]] * ub[ab[1]] for ab in pairs}
    tr = (tau[(0, 0)] + tau[(1, 1)] + tau[(2, 2)]) / 3.0
    T = np.empty((3, 3, M, M, M))
    for (a, b), v in tau.items():
        T[a, b] = T[b, a] = v - (tr if a == b else 0.0)
    axis_of = {0: 2, 1: 1, 2: 0}  # spatial array axis of x, y, z
    g = np.empty((3, 3, M, M, M))  # g[a][b] = d u_b / d x_a
    for a in range(3):
        for b in range(3):
            g[a, b] = 0.5 * (np.roll(ub[b], -1, axis=axis_of[a]) - np.roll(ub[b], 1, axis=axis_of[a]))
    S = 0.5 * (g + g.transpose(1, 0, 2, 3, 4))
    ts = (T * S).sum((0, 1))
    ss = (S * S).sum((0, 1))
    target = np.maximum(0.0, -ts / (2.0 * ss + 1e-30))
    return x, target.reshape(-1)
