"""The 16-bit forms' collision on g = f - w (periodicshiftlbm_b200/csrc/psl_collision_g.cuh),
compiled for the host, against the oracle's cumulant collision (include/applyCollision.h
restated, FP64).  No GPU needed."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "periodicshiftlbm_b200", "csrc")
BUILD = os.path.join(REPO, "tests", "_build")


# D3Q27 weights in the reference's velocity order (include/cellFunctions.h:16)
WEIGHTS = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)


@pytest.fixture(scope="module")
def host_g():
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if not gxx:
        pytest.skip("no host C++ compiler")
    os.makedirs(BUILD, exist_ok=True)
    so = os.path.join(BUILD, "collision_g_host.so")
    subprocess.run([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-shared", "-fPIC", "-I", CSRC,
                    os.path.join(REPO, "tests", "native", "collision_g_host.cpp"), "-o", so], check=True)
    L = ctypes.CDLL(so)
    L.collide_g_host.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_float]
    return L


def _cells(orc, count, seed, amp):
    """Equilibria at random (rho, u) with relative noise of size amp on every population."""
    rng = np.random.default_rng(seed)
    f = np.empty((count, 27))
    for c in range(count):
        rho = 1.0 + rng.uniform(-0.02, 0.02)
        u = rng.uniform(-0.08, 0.08, 3)
        f[c] = orc.feq(rho, *u, dtype=np.float64)
    return f * (1.0 + rng.uniform(-amp, amp, f.shape))


@pytest.mark.parametrize("nu,cs", [(0.008, 0.0), (2.4e-5, 0.1), (1e-5, 0.0), (0.05, 0.2)])
def test_collision_on_deviations_matches_oracle(orc, host_g, nu, cs):
    w = WEIGHTS
    f = _cells(orc, 200, 7, 3e-3)
    g = (f - w).astype(np.float32)
    host_g.collide_g_host(g.ctypes.data, g.shape[0], nu, cs)
    worst_rel, worst_dev = 0.0, 0.0
    for c in range(f.shape[0]):
        want = orc.collision(f[c], nu, cs, dtype=np.float64)
        got = g[c].astype(np.float64) + w
        worst_rel = max(worst_rel, float(np.max(np.abs(got - want) / np.abs(want))))
        # the deviations themselves (what the 16-bit forms store), relative to their size
        worst_dev = max(worst_dev, float(np.max(np.abs(g[c] - (want - w))) / np.max(np.abs(want - w))))
    assert worst_rel < 2e-6, worst_rel
    assert worst_dev < 2e-5, worst_dev


def test_rest_state_is_a_fixed_point(host_g):
    g = np.zeros((1, 27), dtype=np.float32)
    host_g.collide_g_host(g.ctypes.data, 1, 0.01, 0.1)
    # zero up to the FP32 rounding of the weights themselves (ulp(8/27) = 3e-8)
    assert np.max(np.abs(g)) < 1e-7
