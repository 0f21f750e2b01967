"""The grouped thread-to-cell order of the update kernels (psl_rowgroups.cuh), compiled for
the host: the fast division is exact, the order is a permutation of the cells, each group
of 16 x-rows lists its interior cells in cell order and then its x-face cells, and every
x-face warp holds only x-face cells.  No GPU needed."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "periodicshiftlbm_b200", "csrc")
BUILD = os.path.join(REPO, "tests", "_build")


@pytest.fixture(scope="module")
def lib():
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if not gxx:
        pytest.skip("no host C++ compiler")
    os.makedirs(BUILD, exist_ok=True)
    so = os.path.join(BUILD, "rowgroups_host.so")
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC,
                    os.path.join(REPO, "tests", "native", "rowgroups_host.cpp"), "-o", so], check=True)
    L = ctypes.CDLL(so)
    L.fastdiv_host.restype = ctypes.c_uint32
    L.fastdiv_host.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
    L.grouped_cells_host.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
    return L


def test_fast_division_is_exact(lib):
    rng = np.random.default_rng(3)
    divisors = [1, 2, 3, 5, 7, 30, 62, 126, 254, 510, 512, 1022, 4094, 65535, 1 << 20, (1 << 31) + 11, 0xFFFFFFFF]
    xs = np.concatenate([rng.integers(0, 1 << 32, 2000, dtype=np.uint64), [0, 1, 2, (1 << 32) - 1, (1 << 31)]])
    for d in divisors + list(rng.integers(1, 1 << 32, 40, dtype=np.uint64)):
        for x in xs:
            assert lib.fastdiv_host(int(d), int(x)) == int(x) // int(d), (d, x)


@pytest.mark.parametrize("nx,rows", [(4, 1), (8, 5), (16, 16), (16, 17), (34, 40), (512, 48), (256, 33), (6, 100)])
def test_grouped_order_is_a_permutation_with_xface_warps(lib, nx, rows):
    n = nx * rows
    out = np.empty(n, dtype=np.uint32)
    lib.grouped_cells_host(nx, rows, out.ctypes.data)
    assert np.array_equal(np.sort(out), np.arange(n, dtype=np.uint32))
    x = out % nx
    for g0 in range(0, rows, 16):
        r = min(16, rows - g0)
        part = out[g0 * nx:(g0 + r) * nx]
        inner = part[: r * (nx - 2)]
        face = part[r * (nx - 2):]
        assert np.all(np.diff(inner.astype(np.int64)) > 0)           # interior cells in cell order
        assert np.all((inner % nx != 0) & (inner % nx != nx - 1))
        assert np.all((face % nx == 0) | (face % nx == nx - 1))       # then the x-face cells
        assert np.all(face[1:-1:2] + 1 == face[2::2])                 # (row r, Nx-1), (row r+1, 0) adjacent
    if (16 * nx) % 32 == 0 and rows % 16 == 0:  # whole warps: x-face warps hold x-face cells only
        warps = x.reshape(-1, 32)
        face_warp = np.all((warps == 0) | (warps == nx - 1), axis=1)
        inner_warp = np.all((warps != 0) & (warps != nx - 1), axis=1)
        assert np.all(face_warp | inner_warp)
        assert face_warp.sum() == rows // 16
