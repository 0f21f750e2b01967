"""Training of the learned closure on the GPU: the CUDA gradient against the CPU oracle's
FP64 gradient, Adam reducing the loss, the filtered training samples against the oracle's
restatement of the filter, and what the trained closure gains over Smagorinsky."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo
from periodicshiftlbm_b200 import turbulence as tb
from periodicshiftlbm_b200.sgs import Trainer, init_params, mlp_infer, smagorinsky_nu_t

pytestmark = pytest.mark.gpu


def realistic(n, seed):
    rng = np.random.default_rng(seed)
    pi = rng.normal(0.0, 2e-3, (n, 6))
    pxx, pyy, pzz, pxy, pxz, pyz = pi.T
    n2 = pxx ** 2 + pyy ** 2 + pzz ** 2 + 2 * (pxy ** 2 + pxz ** 2 + pyz ** 2)
    det = pxx * (pyy * pzz - pyz * pyz) - pxy * (pxy * pzz - pyz * pxz) + pxz * (pxy * pyz - pyy * pxz)
    return np.column_stack([pi, pxx + pyy + pzz, np.sqrt(n2), det / n2, np.ones(n)])


@pytest.mark.parametrize("count", [1, 100, 128, 5000])
def test_cuda_gradient_matches_fp64_oracle(count):
    x = realistic(6000, 1)
    t = np.random.default_rng(2).uniform(0.0, 0.02, 6000)
    p = mo.random_params(7)
    tr = Trainer(6000)
    tr.add_samples(x, t)
    tr.params = p
    first = 17 if count < 5000 else 0
    loss, g = tr.gradient(first, count)
    p32 = {k: np.asarray(v, dtype=np.float32).astype(np.float64) for k, v in p.items()}
    want_loss, want = mo.loss_and_grad64(p32, x[first:first + count].astype(np.float32),
                                         t[first:first + count].astype(np.float32))
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss)
    for k in want:
        a, b = np.asarray(g[k], np.float64).ravel(), np.asarray(want[k], np.float64).ravel()
        assert np.linalg.norm(a - b) <= 2e-4 * np.linalg.norm(b) + 1e-12, k
    tr.close()


def test_adam_fits_a_learnable_target():
    x = realistic(200_000, 3)
    teacher = mo.random_params(8)
    t = mo.forward64(teacher, x)[-1]
    t = teacher["out_scale"] * mo.softplus(t)
    tr = Trainer(len(t))
    tr.add_samples(x, t)
    p = init_params(x, t, seed=1)
    tr.params = p
    first = tr.gradient(0, 50_000)[0]
    tr.train(600, batch=8192, lr=3e-3, seed=4)
    last = tr.gradient(0, 50_000)[0]
    assert last < 0.1 * first, (first, last)
    tr.close()


def test_filtered_samples_match_oracle(orc):
    M = 6
    fine = tb.box_grid(2 * M, 0.02, cs=0.1)
    tb.fill_from_velocity(fine, tb.initial_velocity(2 * M, seed=5, k0=2.0))
    tb.run(fine, 7)
    tr = Trainer(M ** 3)
    tr.add_filtered(fine, M, stride=1, phase=0)
    x, t = tr.samples()
    want_x, want_t = mo.filtered_samples(fine.fArray, M, lambda f: orc.rescale(f, False))
    # FP32 moments on the GPU vs FP64 (of FP32-rescaled populations) in the oracle
    assert np.max(np.abs(x[:, :6] - want_x[:, :6])) < 5e-7
    assert np.allclose(x[:, 9], 1.0)
    sel = want_t > 1e-3 * want_t.max()
    assert np.median(np.abs(t[sel] - want_t[sel]) / want_t[sel]) < 5e-3
    tr.close()
    fine.close()


def test_trained_closure_beats_smagorinsky_a_priori():
    """The gain of the trained network: on a held-out seed's filtered samples its eddy
    viscosity is closer to the filtered fine run's than Smagorinsky's (C_s = 0.1) and than
    no model at all."""
    M, nu, cs = 16, 2e-4, 0.1
    tr = Trainer(4 * M ** 3)
    for seed in (0, 1):
        fine = tb.box_grid(2 * M, 2 * nu, cs=cs)
        tb.fill_from_velocity(fine, tb.initial_velocity(2 * M, seed, k0=2.0))
        for _ in range(2):
            tb.run(fine, 60)
            tr.add_filtered(fine, M, stride=1, phase=0)
        fine.close()
    x, t = tr.samples()
    tr.params = init_params(x, t, seed=0)
    tr.train(800, batch=4096, lr=2e-3, seed=1)
    p = tr.params
    fine = tb.box_grid(2 * M, 2 * nu, cs=cs)
    tb.fill_from_velocity(fine, tb.initial_velocity(2 * M, 9, k0=2.0))
    tb.run(fine, 90)
    held = Trainer(M ** 3)
    held.add_filtered(fine, M, stride=1, phase=0)
    hx, ht = held.samples()
    pred = mlp_infer(p, hx).astype(np.float64)
    mse_mlp = np.mean((pred - ht) ** 2)
    mse_smag = np.mean((smagorinsky_nu_t(hx, nu, cs) - ht) ** 2)
    mse_zero = np.mean(ht.astype(np.float64) ** 2)
    assert mse_mlp < mse_smag and mse_mlp < mse_zero, (mse_mlp, mse_smag, mse_zero)
    for o in (tr, held, fine):
        o.close()


def test_small_study_runs_end_to_end():
    res = tb.study(M=16, seeds=(0, 1), snapshots=(40, 80), eval_steps=40, nu=2e-4, stride=2, train_steps=200,
                   batch=4096)
    for name, r in res["runs"].items():
        assert r["health"] == 0, name
        assert np.isfinite(r["spectrum_error"]) and r["energy"] > 0, name
    assert res["apriori"]["mse_closure"] < res["apriori"]["mse_zero"]
