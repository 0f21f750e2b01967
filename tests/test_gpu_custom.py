"""The customised update on the GPU (psl_set_body_force, moving-wall and forced-velocity
markers): the forcing scheme's exact momentum gain, and every cell kind against the
reference's moving bounce-back and the oracle's forcing collision."""
import numpy as np
import pytest

from gpu_helpers import rel
from oracle import mlp_oracle as mo
from periodicshiftlbm_b200 import (
    GridStruct,
    InfoStruct,
    _lib,
    applyLocalCellUpdate,
    applyStreaming,
    fillEquilibriumFromFunction,
    setBodyForce,
)
from periodicshiftlbm_b200.grid import MARKER_FORCED_VELOCITY, MARKER_MOVING_WALL
from periodicshiftlbm_b200.sgs import set_sgs_mlp

pytestmark = pytest.mark.gpu

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1])
CZ = np.array([0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1])


def noisy_grid(n=(12, 10, 8), nu=0.02, seed=0):
    g = GridStruct(InfoStruct(cellCountX=n[0], cellCountY=n[1], cellCountZ=n[2], nu=nu))
    fillEquilibriumFromFunction(g, rho=1.0, u=(0.02, -0.01, 0.005))
    f = g.fArray
    f *= (1.0 + np.random.default_rng(seed).uniform(-1e-2, 1e-2, f.shape)).astype(np.float32)
    g.fArray = f
    return g


def test_body_force_adds_g_per_cell_and_step():
    g = noisy_grid()
    j0 = np.array([(c[:, None] * g.fArray.astype(np.float64)).sum() for c in (CX, CY, CZ)])
    force = (1e-4, -2e-5, 0.0)
    setBodyForce(g, *force)
    steps = 10
    for _ in range(steps):
        applyStreaming(g)
        applyLocalCellUpdate(g)
    j1 = np.array([(c[:, None] * g.fArray.astype(np.float64)).sum() for c in (CX, CY, CZ)])
    expected = np.array(force) * steps * g.cellCount
    # exact in exact arithmetic; each step rounds every stored population to FP32 (about
    # 1e-9 per cell and step against a force of 1e-4)
    assert abs((j1 - j0)[0] - expected[0]) < 1e-3 * abs(expected[0])
    assert abs((j1 - j0)[1] - expected[1]) < 1e-3 * abs(expected[0])
    assert abs((j1 - j0)[2]) < 1e-3 * abs(expected[0])
    assert g.health() == 0
    g.close()


def test_customised_update_matches_reference_and_oracle(ref, orc):
    nu, body = 0.02, (3e-6, 1e-6, -2e-6)
    g = noisy_grid(nu=nu, seed=1)
    n = g.cellCount
    rng = np.random.default_rng(4)
    markers = np.full(n, _lib.CELL_FLUID, dtype=np.uint8)
    kind = rng.choice(4, n, p=[0.55, 0.15, 0.15, 0.15])  # fluid, forced, moving wall, solid
    markers[kind == 1] = MARKER_FORCED_VELOCITY
    markers[kind == 2] = MARKER_MOVING_WALL
    markers[kind == 3] = _lib.CELL_SOLID
    given = np.zeros((n, 4), dtype=np.float32)
    given[:, 0] = 1.0
    given[:, 1:] = rng.uniform(-0.05, 0.05, (n, 3)).astype(np.float32)
    g.markers = markers
    from periodicshiftlbm_b200._lib import call

    call("psl_set_given_field", g.handle, np.ascontiguousarray(given).ctypes.data)
    setBodyForce(g, *body)
    applyStreaming(g)
    f_in = g.fArray
    applyLocalCellUpdate(g)
    f_out = g.fArray
    assert g.health() == 0
    for c in range(n):
        fi = f_in[:, c]
        if kind[c] == 2:  # moving wall: the reference's own function, bit for bit
            want = ref.moving_bounceback(fi, *given[c, 1:])
            assert np.array_equal(f_out[:, c], want), c
        elif kind[c] == 3:
            want = fi.copy()
            want[1::2], want[2::2] = fi[2::2], fi[1::2]
            assert np.array_equal(f_out[:, c], want), c
        else:
            gx, gy, gz = (np.float32(v) for v in body)
            if kind[c] == 1:
                f64 = fi.astype(np.float64)
                rho = f64.sum()
                u = np.array([(CX * f64).sum(), (CY * f64).sum(), (CZ * f64).sum()]) / rho
                d = rho * (given[c, 1:].astype(np.float64) - u)
                gx, gy, gz = gx + d[0], gy + d[1], gz + d[2]
            want = orc.collision(fi, nu, 0.0, force=(float(gx), float(gy), float(gz)))
            assert rel(f_out[:, c], want) < 2e-6, c
    g.close()


def test_learned_closure_refuses_forcing():
    g = noisy_grid()
    set_sgs_mlp(g, mo.random_params(1), 1.0)
    setBodyForce(g, 1e-6, 0.0, 0.0)
    applyStreaming(g)
    with pytest.raises(_lib.PslError):
        applyLocalCellUpdate(g)
    g.close()
