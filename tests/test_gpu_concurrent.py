"""psl_update_grid's concurrent schedule against the serial one.

For a refined hierarchy psl_update_grid updates the coarse cells away from the refinement
block on a side stream beside the fine updates and the transfer.  No cell's data is
touched by both, so every population and every drag must equal, bit for bit, those of the
same steps issued one call at a time (applyStreaming, applyLocalCellUpdate, the fine
recursion, applyCoarseFineGridCommunication: one launch after another on one stream)."""
import dataclasses

import numpy as np
import pytest

from oracle import mlp_oracle as mo
from periodicshiftlbm_b200 import (applyCoarseFineGridCommunication, applyLocalCellUpdate, applyStreaming,
                                   updateGrid)
from periodicshiftlbm_b200.cases import config2, make_sphere_grids
from periodicshiftlbm_b200.grid import getSphereDrag
from periodicshiftlbm_b200.sgs import set_sgs_mlp

pytestmark = pytest.mark.gpu


def serial_step(grids, level=0):
    g = grids[level]
    applyStreaming(g)
    applyLocalCellUpdate(g)
    if level < len(grids) - 1:
        serial_step(grids, level + 1)
        serial_step(grids, level + 1)
        applyCoarseFineGridCommunication(g, grids[level + 1])


@pytest.mark.parametrize("storage,closure", [("f32", None), ("f16", None), ("bf16", None), ("f16", 4)])
def test_concurrent_schedule_equals_serial(storage, closure):
    cfg = config2(scale=0.5)
    runs = []
    for concurrent in (True, False):
        grids, case = make_sphere_grids(cfg, storage=storage)
        if closure:
            p = mo.random_params(11)
            for g in grids:
                set_sgs_mlp(g, p, filter_width=g.Info.res / grids[0].Info.res, interval=closure)
        drags = []
        for _ in range(9):
            if concurrent:
                updateGrid(grids, 0)
            else:
                serial_step(grids)
            drags.append(getSphereDrag(grids[-1], case))
        runs.append(([g.fArray for g in grids], [g.shifter for g in grids], drags, [g.health() for g in grids]))
        for g in grids:
            g.close()
    (fa, sa, da, ha), (fb, sb, db, hb) = runs
    for lvl in range(2):
        assert np.array_equal(sa[lvl], sb[lvl])
        assert np.array_equal(fa[lvl], fb[lvl]), (lvl, np.abs(fa[lvl] - fb[lvl]).max())
    assert da == db
    assert ha == hb == [0, 0]


def test_concurrent_schedule_three_levels():
    """A three-level hierarchy: the top pair runs concurrently, the inner pair serially."""
    cfg = dataclasses.replace(config2(scale=0.25), refine2=((8, 8, 8), (56, 40, 40)))  # level-1 cells
    runs = []
    for concurrent in (True, False):
        grids, case = make_sphere_grids(cfg)
        assert len(grids) == 3
        for _ in range(4):
            updateGrid(grids, 0) if concurrent else serial_step(grids)
        runs.append([g.fArray for g in grids])
        for g in grids:
            assert g.health() == 0
            g.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)
