"""The learned subgrid closure on the tensor cores (tcgen05 + TMEM), checked against the CPU
oracle (oracle/mlp_oracle.py) and against the plain update kernel."""
import numpy as np
import pytest

from gpu_helpers import rel
from oracle import mlp_oracle as mo
from periodicshiftlbm_b200 import GridStruct, InfoStruct, applyLocalCellUpdate, applyStreaming, fillEquilibriumFromFunction
from periodicshiftlbm_b200.sgs import mlp_infer, set_sgs_mlp, set_sgs_mlp_interval

pytestmark = pytest.mark.gpu


def realistic_features(n, seed):
    rng = np.random.default_rng(seed)
    pi = rng.normal(0.0, 2e-3, (n, 6))
    pxx, pyy, pzz, pxy, pxz, pyz = pi.T
    n2 = pxx ** 2 + pyy ** 2 + pzz ** 2 + 2 * (pxy ** 2 + pxz ** 2 + pyz ** 2)
    det = pxx * (pyy * pzz - pyz * pyz) - pxy * (pxy * pzz - pyz * pxz) + pxz * (pxy * pyz - pyy * pxz)
    return np.column_stack([pi, pxx + pyy + pzz, np.sqrt(n2), det / n2, np.ones(n)]).astype(np.float32)


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 4096])
def test_tensor_core_inference_matches_oracle(n):
    p = mo.random_params(3)
    x = realistic_features(n, n)
    got = mlp_infer(p, x)
    want = mo.forward_device(p, x)
    # FP16 operands and FP32 accumulation on both sides; only the summation order differs
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-6)) < 2e-3


def test_inference_is_not_a_constant():
    """Guards against a path that ignores its inputs (e.g. an MMA that never ran)."""
    p = mo.random_params(4)
    x = realistic_features(512, 9)
    got = mlp_infer(p, x)
    assert np.std(got) > 0.05 * np.mean(np.abs(got))


def periodic_grid(storage="f32", n=(16, 12, 10), nu=0.01, seed=1):
    g = GridStruct(InfoStruct(cellCountX=n[0], cellCountY=n[1], cellCountZ=n[2], nu=nu), storage=storage)
    fillEquilibriumFromFunction(g, rho=1.0, u=(0.03, -0.01, 0.02))
    rng = np.random.default_rng(seed)
    f = g.fArray
    f *= (1.0 + rng.uniform(-2e-2, 2e-2, f.shape)).astype(np.float32)
    g.fArray = f
    return g


# grid shapes: whole 128-cell blocks and wrap points at block edges (16x12x10 = 15 blocks)
# or a partial last block (15x11x9)
SHAPES = {"whole": (16, 12, 10), "partial": (15, 11, 9)}


@pytest.mark.parametrize("path", ["whole", "partial"])
def test_constant_closure_equals_plain_update_with_added_viscosity(path):
    _constant_closure_check(SHAPES[path])


def _constant_closure_check(shape):
    p = {k: np.zeros_like(v) for k, v in mo.random_params(0).items()}
    p["in_scale"] = np.ones(10)
    p["b3"] = np.float64(0.3)
    p["out_scale"] = np.float64(0.004)
    nu_t = float(mlp_infer(p, np.zeros((1, 10), np.float32))[0])
    a = periodic_grid(n=shape, nu=0.01)
    b = periodic_grid(n=shape, nu=float(np.float32(0.01) + np.float32(nu_t)))
    set_sgs_mlp(a, p, 1.0)
    for _ in range(5):
        for g in (a, b):
            applyStreaming(g)
            applyLocalCellUpdate(g)
    assert rel(a.fArray, b.fArray) < 1e-6
    assert a.health() == 0
    a.close()
    b.close()


@pytest.mark.parametrize("path", ["whole", "partial"])
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_fused_learned_update_matches_oracle_cell_by_cell(orc, storage, path):
    """The fused closure on every storage form, whole and partial blocks."""
    p = mo.random_params(5)
    g = periodic_grid(storage=storage, n=SHAPES[path], nu=0.01)
    set_sgs_mlp(g, p, 1.0)
    applyStreaming(g)
    f_in = g.fArray  # the populations each cell loads
    applyLocalCellUpdate(g)
    f_out = g.fArray
    assert g.health() == 0
    x = mo.features(f_in, 1.0)
    nu_t = mo.forward_device(p, x.astype(np.float32))
    assert np.std(nu_t) > 0
    idx = np.random.default_rng(0).choice(f_in.shape[1], 300, replace=False)
    want = np.stack([orc.collision(f_in[:, c], float(np.float32(0.01) + nu_t[c]), 0.0) for c in idx], axis=1)
    if storage == "f32":
        assert rel(f_out[:, idx], want) < 1e-5
    else:  # the result is stored as 16-bit f - w
        w = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)[:, None]
        bound = 2e-3 if storage == "f16" else 1.6e-2
        assert np.max(np.abs(f_out[:, idx] - want) / np.maximum(np.abs(want - w), 1e-4)) < bound
    g.close()


W_LATTICE = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)[:, None]


def _check_against_oracle(orc, storage, f_in, f_out, nu_t, idx):
    """f_out[:, idx] is the oracle collision of f_in[:, idx] at viscosity 0.01 + nu_t, within
    the bound of the stored 16-bit f - w (as the fused-update test)."""
    want = np.stack([orc.collision(f_in[:, c], float(np.float32(0.01) + np.float32(nu_t[c])), 0.0) for c in idx],
                    axis=1)
    bound = 2e-3 if storage == "f16" else 1.6e-2
    err = np.max(np.abs(f_out[:, idx] - want) / np.maximum(np.abs(want - W_LATTICE), 1e-4))
    assert err < bound, err


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_closure_interval_first_update_equals_every_update(storage):
    """With an interval the first update still runs the network: the same bits as the
    closure on every update."""
    p = mo.random_params(5)
    a = periodic_grid(storage=storage)
    b = periodic_grid(storage=storage)
    set_sgs_mlp(a, p, 1.0)
    set_sgs_mlp(b, p, 1.0, interval=3)
    for g in (a, b):
        applyStreaming(g)
        applyLocalCellUpdate(g)
    assert np.array_equal(a.fArray, b.fArray)
    for g in (a, b):
        assert g.health() == 0
        g.close()


@pytest.mark.parametrize("path", ["whole", "partial"])
@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_closure_interval_updates_use_the_kept_nu_t(orc, storage, path):
    """Interval 3: updates 1 and 4 run the network on their own input; updates 2 and 3
    relax with the nu_t of update 1's input, kept in FP16."""
    p = mo.random_params(5)
    g = periodic_grid(storage=storage, n=SHAPES[path], nu=0.01)
    set_sgs_mlp(g, p, 1.0, interval=3)
    idx = np.random.default_rng(1).choice(g.cellCount, 200, replace=False)
    kept = None
    for step in range(4):
        applyStreaming(g)
        f_in = g.fArray
        applyLocalCellUpdate(g)
        f_out = g.fArray
        if step % 3 == 0:
            nu_t = mo.forward_device(p, mo.features(f_in, 1.0).astype(np.float32))
            kept = nu_t.astype(np.float16).astype(np.float32)
        else:
            nu_t = kept
        _check_against_oracle(orc, storage, f_in, f_out, nu_t, idx)
    assert g.health() == 0
    g.close()


def test_closure_interval_restarts_after_new_populations():
    """Setting populations from outside makes the next update run the network again."""
    p = mo.random_params(7)
    a = periodic_grid(storage="f16", seed=3)
    b = periodic_grid(storage="f16", seed=3)
    set_sgs_mlp(a, p, 1.0, interval=4)
    set_sgs_mlp(b, p, 1.0)
    applyStreaming(a)
    applyLocalCellUpdate(a)           # runs the network; the next three would not
    b.shifter = a.shifter             # both at the same shifts and state
    b.fArray = a.fArray
    a.fArray = a.fArray               # a fresh state set from outside
    for g in (a, b):
        applyStreaming(g)
        applyLocalCellUpdate(g)
    assert np.array_equal(a.fArray, b.fArray)
    set_sgs_mlp_interval(a, 1)        # back to every update: the kept field is released
    for g in (a, b):
        applyStreaming(g)
        applyLocalCellUpdate(g)
    assert np.array_equal(a.fArray, b.fArray)
    a.close()
    b.close()


def test_closure_interval_needs_16_bit_storage():
    g = periodic_grid(storage="f32")
    with pytest.raises(Exception, match="FP16 or BF16"):
        set_sgs_mlp_interval(g, 2)
    with pytest.raises(Exception, match="at least 1"):
        set_sgs_mlp_interval(g, 0)
    set_sgs_mlp_interval(g, 1)
    g.close()


def test_closure_can_be_removed():
    p = mo.random_params(6)
    a = periodic_grid()
    b = periodic_grid()
    set_sgs_mlp(a, p, 1.0)
    set_sgs_mlp(a, None)
    for g in (a, b):
        applyStreaming(g)
        applyLocalCellUpdate(g)
    assert np.array_equal(a.fArray, b.fArray)
    a.close()
    b.close()
