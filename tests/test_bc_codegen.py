"""The boundary-condition generator (periodicshiftlbm_b200/csrc/gen_bc.py): its committed
output is current, and the emitted CUDA code, compiled for the host, reproduces the
reference's boundary functions bit for bit.  No GPU needed."""
import importlib.util
import os
import shutil
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "periodicshiftlbm_b200", "csrc")
BUILD = os.path.join(REPO, "tests", "_build")


def _gen_module():
    spec = importlib.util.spec_from_file_location("gen_bc", os.path.join(CSRC, "gen_bc.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_generated_files_are_current():
    gen = _gen_module()
    meq = gen.equilibrium_moments()
    qlin = [gen.linear_part(e) for e in meq]
    bcs = [gen.NormalBC(n, meq, qlin) for n in gen.NORMALS]
    with open(gen.CUDA_OUT) as fh:
        assert fh.read() == gen.emit_cuda(bcs)
    with open(gen.ORACLE_OUT) as fh:
        assert fh.read() == gen.emit_oracle(bcs, meq)


def test_unknown_sets_follow_outer_normal():
    gen = _gen_module()
    meq = gen.equilibrium_moments()
    qlin = [gen.linear_part(e) for e in meq]
    counts = {}
    for n in gen.NORMALS:
        b = gen.NormalBC(n, meq, qlin)
        counts.setdefault(sum(abs(c) for c in n), set()).add(len(b.unknown))
        # every mirror source is a known population
        assert all(src in b.known for src in b.mirror.values())
    assert counts == {1: {9}, 2: {15}, 3: {19}}


@pytest.fixture(scope="module")
def host_bc():
    import ctypes

    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if not gxx:
        pytest.skip("no host C++ compiler")
    os.makedirs(BUILD, exist_ok=True)
    so = os.path.join(BUILD, "bc_host_check.so")
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC,
                    os.path.join(REPO, "tests", "native", "bc_host_check.cpp"), "-o", so], check=True)
    L = ctypes.CDLL(so)
    L.bc_host.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return L


def test_generated_bc_bitwise_equals_reference(host_bc):
    g = np.load(os.path.join(REPO, "tests", "golden", "cell_functions.npz"))
    F = g["f_in"]
    for a, nrm in enumerate(g["bc_normals"]):
        idx = (int(nrm[0]) + 1) * 9 + (int(nrm[1]) + 1) * 3 + (int(nrm[2]) + 1)
        for i in range(F.shape[0]):
            rho = g["bc_rho"][a, i]
            u = g["bc_u"][a, i]

            def run(op, args):
                v = F[i].copy()
                arr = np.array(args, dtype=np.float32)
                host_bc.bc_host(op, idx, v.ctypes.data, arr.ctypes.data)
                return v

            assert np.array_equal(run(2, [rho, *u]), g["mbbc_out"][a, i]), tuple(nrm)
            assert run(3, [1.0, *u])[0] == g["restore_rho_out"][a, i]
            assert np.array_equal(run(4, [rho, 0, 0, 0])[:3], g["restore_u_out"][a, i])
            assert np.array_equal(run(5, [1.0, 0, 0, 0])[:4], g["restore_rho_u_out"][a, i])
            assert np.array_equal(run(6, [0, 0, 0, 0]), g["mirror_out"][a, i])
