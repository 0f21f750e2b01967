"""Host-side check of the tiled update kernel's index arithmetic (psl_step_tiled.cuh):
for every block and population row, the bulk loads stay inside the row and inside the
shared buffer, respect the 16-byte rules, and the write-back covers every address of the
row exactly once.  Mirrors the kernel's integer math; no GPU needed."""
import numpy as np
import pytest

TILE = 128


def plan(n, shift, c0, V):
    """(loads, smem_off, writes) of one block for one row, as the kernel computes them.
    loads: [(global_start, n_elems, smem_dst)], writes: [(g0, g1, smem_start, h0, h1)]"""
    a = c0 + shift
    if a >= n:
        a -= n
    a0 = a & ~(V - 1)
    off = a - a0
    loads = []
    if a + TILE <= n:
        a1 = (a + TILE + V - 1) & ~(V - 1)
        loads.append((a0, a1 - a0, 0))
    else:
        loads.append((a0, n - a0, 0))
        rest = (a + TILE - n + V - 1) & ~(V - 1)
        loads.append((0, rest, n - a0))
    segs = [(a, a + TILE, off)] if a + TILE <= n else [(a, n, off), (0, a + TILE - n, off + (n - a))]
    writes = []
    for g0, g1, s in segs:
        h0 = (g0 + V - 1) & ~(V - 1)
        h1 = g1 & ~(V - 1)
        writes.append((g0, g1, s, h0, h1))
    return loads, off, writes


@pytest.mark.parametrize("elem_bytes", [4, 2])
@pytest.mark.parametrize("dims", [(16, 8, 8), (128, 64, 64), (24, 16, 16), (256, 3, 7)])
def test_tile_plan_in_bounds_aligned_and_covering(elem_bytes, dims):
    V = 16 // elem_bytes
    R = TILE + 2 * V
    n = dims[0] * dims[1] * dims[2]
    if n % TILE:
        pytest.skip("tiled kernel requires N % 128 == 0")
    rng = np.random.default_rng(n + elem_bytes)
    for trial in range(20):
        shift = int(rng.integers(0, n)) if trial else 0
        covered = np.zeros(n, dtype=np.int32)
        for c0 in range(0, n, TILE):
            loads, off, writes = plan(n, shift, c0, V)
            for start, count, dst in loads:
                assert count > 0 and start >= 0 and start + count <= n  # inside the row
                assert (start * elem_bytes) % 16 == 0 and (count * elem_bytes) % 16 == 0
                assert (dst * elem_bytes) % 16 == 0 and dst + count <= R  # inside the shared row
            # every thread's element index is inside the loaded cover
            loaded = np.zeros(R, dtype=bool)
            for start, count, dst in loads:
                loaded[dst:dst + count] = True
            assert loaded[off:off + TILE].all()
            for g0, g1, s, h0, h1 in writes:
                assert 0 <= g0 < g1 <= n
                if h1 > h0:
                    assert ((s + h0 - g0) * elem_bytes) % 16 == 0  # bulk-store source aligned
                    assert (h0 * elem_bytes) % 16 == 0 and ((h1 - h0) * elem_bytes) % 16 == 0
                assert s + (g1 - g0) <= R
                covered[g0:g1] += 1
        assert np.all(covered == 1)
