"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Runs oracle/_ref/libpsl_ref.so -- the reference project's headers compiled unmodified for
the host (oracle/ref_cases.cpp, oracle/Makefile) -- on seeded synthetic inputs and saves
its outputs.  Needs the reference checkout to have been built into oracle/_ref; the saved
fixtures are what the tests use on machines without it.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle.bindings import ALL_NORMALS, RefLib, SphereCase  # noqa: E402

# Small sphere runs (coarse-cell units).  Steps are kept short enough to generate quickly.
RUNS = {
    "tiny_mirror": dict(case=SphereCase(nx=12, ny=8, nz=8, sphere=(4.0, 4.0, 4.0), radius=1.5, nu=0.02), steps=60,
                        full=True),
    "small_velwall_les": dict(case=SphereCase(nx=24, ny=16, nz=16, sphere=(8.0, 8.0, 8.0), radius=3.0, nu=0.001,
                                              smagorinsky=0.1, wall_mode=1), steps=100, full=False),
    "small_refined_les": dict(case=SphereCase(nx=32, ny=16, nz=16, sphere=(14.0, 8.0, 8.0), radius=2.5, nu=0.005,
                                              smagorinsky=0.1, refine=((8, 4, 4), (20, 12, 12))), steps=40, full=False),
    "config1_1000": dict(case=SphereCase(), steps=1000, full=False),
}
N_SAMPLE = 2048


def sample_cells(n: int, seed: int = 7) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=min(n, N_SAMPLE), replace=False))


def cell_function_vectors(R: RefLib) -> dict:
    """Single-function inputs/outputs of the reference's device functions."""
    rng = np.random.default_rng(2024)
    n = 64
    out = {}
    fs = []
    for _ in range(n):
        u = rng.uniform(-0.08, 0.08, 3)
        rho = 1.0 + rng.uniform(-0.03, 0.03)
        fe = R.feq(rho, *u)
        fs.append((fe * (1.0 + rng.uniform(-0.05, 0.05, 27))).astype(np.float32))
    F = np.stack(fs)
    out["f_in"] = F
    params = [(0.008, 0.0), (2.4e-5, 0.1), (0.001, 0.1)]
    out["collision_params"] = np.array(params, dtype=np.float32)
    out["collision_out"] = np.stack([np.stack([R.collision(f, nu, cs) for f in F]) for nu, cs in params])
    out["rescale_c2f"] = np.stack([R.rescale(f, True) for f in F])
    out["rescale_f2c"] = np.stack([R.rescale(f, False) for f in F])
    bc_args = rng.uniform(-0.05, 0.05, (len(ALL_NORMALS), n, 3)).astype(np.float32)
    bc_rho = (1.0 + rng.uniform(-0.02, 0.02, (len(ALL_NORMALS), n))).astype(np.float32)
    out["bc_normals"] = np.array(ALL_NORMALS, dtype=np.int32)
    out["bc_u"] = bc_args
    out["bc_rho"] = bc_rho
    mb, rr, ru, rru, mi = [], [], [], [], []
    for a, nrm in enumerate(ALL_NORMALS):
        mb.append(np.stack([R.mbbc(nrm, bc_rho[a, i], *bc_args[a, i], F[i]) for i in range(n)]))
        rr.append(np.array([R.restore_rho(nrm, *bc_args[a, i], F[i]) for i in range(n)], dtype=np.float32))
        ru.append(np.stack([R.restore_u(nrm, bc_rho[a, i], F[i]) for i in range(n)]))
        rru.append(np.stack([R.restore_rho_u(nrm, F[i]) for i in range(n)]))
        mi.append(np.stack([R.mirror(nrm, F[i]) for i in range(n)]))
    out["mbbc_out"] = np.stack(mb)
    out["restore_rho_out"] = np.stack(rr)
    out["restore_u_out"] = np.stack(ru)
    out["restore_rho_u_out"] = np.stack(rru)
    out["mirror_out"] = np.stack(mi)
    out["bounceback_out"] = np.stack([R.bounceback(f) for f in F])
    out["moving_bb_u"] = np.array([0.01, -0.02, 0.03], dtype=np.float32)
    out["moving_bb_out"] = np.stack([R.moving_bounceback(f, 0.01, -0.02, 0.03) for f in F])
    shifts = {}
    for dims in [(8, 6, 5), (128, 64, 64), (7, 3, 1), (256, 192, 192)]:
        s = np.zeros(27, dtype=np.int32)
        seq = []
        for _ in range(5):
            s = R.streaming(dims, s)
            seq.append(s.copy())
        shifts[dims] = np.stack(seq)
    out["stream_dims"] = np.array(list(shifts.keys()), dtype=np.int32)
    out["stream_shifts"] = np.stack(list(shifts.values()))
    return out


def main():
    R = RefLib()
    np.savez_compressed(os.path.join(HERE, "cell_functions.npz"), **cell_function_vectors(R))
    print("wrote cell_functions.npz")
    for name, spec in RUNS.items():
        case = spec["case"]
        sim = R.sim(case)
        sim.run(spec["steps"])
        rec = {"steps": np.int32(spec["steps"]), "drag": np.float64(sim.drag())}
        for lev in range(sim.levels):
            f = sim.populations(lev)
            rec[f"shifts_{lev}"] = sim.shifts(lev)
            rec[f"checksum_{lev}"] = f.astype(np.float64).sum(axis=1)
            if spec["full"]:
                rec[f"f_{lev}"] = f
            else:
                idx = sample_cells(f.shape[1], seed=7 + lev)
                rec[f"sample_idx_{lev}"] = idx.astype(np.int64)
                rec[f"sample_f_{lev}"] = f[:, idx]
        np.savez_compressed(os.path.join(HERE, f"run_{name}.npz"), **rec)
        print(f"wrote run_{name}.npz (drag {rec['drag']:.6g})")


if __name__ == "__main__":
    main()
