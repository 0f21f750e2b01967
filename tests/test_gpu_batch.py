"""Batched form on the GPU: one persistent kernel per step over many grids, replayed from a
CUDA graph, must give each grid exactly the state its own solo run gives."""
import numpy as np
import pytest

from periodicshiftlbm_b200 import _lib, applyStreaming, getSphereDrag, updateGrid
from periodicshiftlbm_b200.batch import Batch, make_batch_grids
from periodicshiftlbm_b200.cases import SphereConfig, make_sphere_grids

pytestmark = pytest.mark.gpu


def small_configs():
    out = []
    for i, (x, re) in enumerate([(16, 100.0), (24, 3e3), (32, 1e5), (24, 400.0), (16, 1e6)]):
        y = x // 2
        d = x / 8.0
        out.append(SphereConfig(name=f"t{i}", nx=x, ny=y, nz=y, sphere=(x / 4, y / 2, y / 2), radius=d / 2,
                                u_in=0.05, nu=0.05 * d / re, smagorinsky=0.1 if re > 1e3 else 0.0, seed=7 + i))
    return out


def solo_state(cfg, steps, storage="f32"):
    grids, case = make_sphere_grids(cfg, storage=storage)
    for _ in range(steps):
        updateGrid(grids, 0)
    out = (grids[0].fArray, grids[0].shifter, getSphereDrag(grids[0], case))
    grids[0].close()
    return out


@pytest.mark.parametrize("tuning", [None, {"threads": 64, "tile_cells": 64, "blocks_per_sm": 4},
                                    {"threads": 256, "tile_cells": 1024, "blocks_per_sm": 2},
                                    {"threads": 128, "tile_cells": 96, "blocks_per_sm": 3},
                                    {"threads": 128, "tile_cells": 64, "blocks_per_sm": 0}])
def test_batched_equals_solo_runs(tuning):
    cfgs = small_configs()
    grids, cases = make_batch_grids(cfgs)
    b = Batch(grids)
    if tuning:
        b.tuning = tuning
    b.run(7)
    b.run(13)  # a second run continues from the device step counter
    for cfg, g, c in zip(cfgs, grids, cases):
        f, s, d = solo_state(cfg, 20)
        assert np.array_equal(g.shifter, s), cfg.name
        assert np.array_equal(g.fArray, f), cfg.name
        assert getSphereDrag(g, c) == d
        assert g.health() == 0
    b.close()
    for g in grids:
        g.close()


def test_autotune_keeps_state_and_picks_a_valid_shape():
    cfgs = small_configs()
    grids, _ = make_batch_grids(cfgs)
    b = Batch(grids)
    b.run(3)
    before = [g.fArray for g in grids]
    t = b.autotune(2)
    assert t["ms_per_step"] > 0 and t["tile_cells"] % 32 == 0 and t["threads"] % 32 == 0
    for g, f in zip(grids, before):
        assert np.array_equal(g.fArray, f)
    b.run(5)
    for cfg, g in zip(cfgs, grids):
        f, s, _ = solo_state(cfg, 8)
        assert np.array_equal(g.fArray, f), cfg.name
    b.close()
    for g in grids:
        g.close()


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_batched_16bit_storage_equals_solo_runs(storage):
    """The 16-bit f - w forms batch like FP32: each grid bit for bit as its own run."""
    cfgs = small_configs()[:3]
    grids, cases = make_batch_grids(cfgs, storage=storage)
    b = Batch(grids)
    b.tuning = {"threads": 128, "tile_cells": 64, "blocks_per_sm": 0}
    b.run(9)
    for cfg, g, c in zip(cfgs, grids, cases):
        f, s, d = solo_state(cfg, 9, storage)
        assert np.array_equal(g.shifter, s), cfg.name
        assert np.array_equal(g.fArray, f), cfg.name
        assert getSphereDrag(g, c) == d
    b.close()
    for g in grids:
        g.close()


def test_batch_guards_member_grids():
    cfgs = small_configs()[:2]
    grids, _ = make_batch_grids(cfgs)
    b = Batch(grids)
    with pytest.raises(_lib.PslError):
        grids[0].close()  # destroy refuses a member grid
    applyStreaming(grids[1])  # streamed outside the batch
    with pytest.raises(_lib.PslError):
        b.run(1)
    b.close()
    for g in grids:
        g.close()


def test_batch_rejects_mixed_storage():
    a, _ = make_sphere_grids(small_configs()[0])
    c, _ = make_sphere_grids(small_configs()[1], storage="f16")
    with pytest.raises(_lib.PslError):
        Batch([a[0], c[0]])
    a[0].close()
    c[0].close()
