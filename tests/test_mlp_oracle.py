"""The CPU oracle of the learned closure, pinned by finite differences (no GPU)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences():
    p = mo.random_params(11)
    rng = np.random.default_rng(2)
    x = rng.normal(0.0, 2e-3, (64, 10))
    x[:, 9] = 1.0
    t = rng.uniform(0.0, 0.02, 64)
    loss, g = mo.loss_and_grad64(p, x, t)
    eps = 1e-6
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        flat = np.asarray(p[name], dtype=np.float64).reshape(-1)
        for i in rng.choice(flat.size, min(6, flat.size), replace=False):
            q = {k: np.array(v, dtype=np.float64, copy=True) for k, v in p.items()}
            fq = q[name].reshape(-1)
            fq[i] += eps
            q[name] = fq.reshape(np.shape(p[name]))
            lp, _ = mo.loss_and_grad64(q, x, t)
            fq[i] -= 2 * eps
            q[name] = fq.reshape(np.shape(p[name]))
            lm, _ = mo.loss_and_grad64(q, x, t)
            num = (lp - lm) / (2 * eps)
            ana = np.asarray(g[name]).reshape(-1)[i]
            assert abs(num - ana) <= 1e-5 * max(1.0, abs(num)), (name, i, num, ana)


def test_device_forward_emulation_tracks_fp64():
    p = mo.random_params(12)
    rng = np.random.default_rng(3)
    x = rng.normal(0.0, 2e-3, (256, 10))
    x[:, 9] = 1.0
    z = mo.forward64(p, x)[-1]
    exact = p["out_scale"] * mo.softplus(z)
    dev = mo.forward_device(p, x.astype(np.float32))
    assert np.max(np.abs(dev - exact) / np.abs(exact)) < 2e-2  # FP16 operands


def test_features_of_equilibrium_are_zero_stress():
    # feq has Pi = u u (per unit density); at rest Pi = 0
    w = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
    x = mo.features(w[:, None], 0.5)
    assert np.allclose(x[0, :9], 0.0, atol=1e-15) and x[0, 9] == 0.5
