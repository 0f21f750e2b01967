"""Host-side check of the pipelined update kernel's index arithmetic
(periodicshiftlbm_b200/csrc/psl_step_pipe.cuh), mirroring its integer math: for every tile
and population row, the bulk loads stay inside the row and the stage's shared row and obey
the 16-byte rules; every cell's element lies in the loaded cover at rem_q + t; the
write-back (head pieces, aligned bulk interior, tail pieces) is aligned, writes only the
tile's own run, and covers every element of the row exactly once over all tiles; the
byte count the kernel arms its mbarrier with equals the bytes it copies.  No GPU needed."""
import numpy as np
import pytest

TILE = 128


def loads_of(n, shift, c0, V):
    """[(global_start, n_elems, smem_dst_elem)] of one row, as pipe_issue_loads computes them."""
    L = min(TILE, n - c0)
    a = c0 + shift
    if a >= n:
        a -= n
    a0 = a & ~(V - 1)
    if a + L <= n:
        return a, a0, [(a0, ((a + L + V - 1) & ~(V - 1)) - a0, 0)]
    return a, a0, [(a0, n - a0, 0), (0, (a + L - n + V - 1) & ~(V - 1), n - a0)]


def segment_pieces(g0, g1, x0, V, E):
    """[(global_elem, n_elems, smem_elem, kind)] written by pipe_write_segment."""
    M = 1 << 32
    sp = lambda x: (x - x0) % M  # noqa: E731  (uint32 arithmetic of the kernel)
    h0 = (g0 + V - 1) & ~(V - 1)
    h1 = g1 & ~(V - 1)
    out = []
    if h1 <= h0:
        return [(x, 1, sp(x), "elem") for x in range(g0, g1)]
    x = g0
    if E == 2 and (x & 1):
        out.append((x, 1, sp(x), "piece")); x += 1
    if x & (4 // E):
        out.append((x, 4 // E, sp(x), "piece")); x += 4 // E
    if x & (8 // E):
        out.append((x, 8 // E, sp(x), "piece")); x += 8 // E
    assert x == h0
    out.append((h0, h1 - h0, sp(h0), "bulk"))
    x = h1
    r = g1 - h1
    if r & (8 // E):
        out.append((x, 8 // E, sp(x), "piece")); x += 8 // E
    if r & (4 // E):
        out.append((x, 4 // E, sp(x), "piece")); x += 4 // E
    if E == 2 and (r & 1):
        out.append((x, 1, sp(x), "piece")); x += 1
    assert x == g1
    return out


def stores_of(n, shift, c0, V, E):
    L = min(TILE, n - c0)
    a = c0 + shift
    if a >= n:
        a -= n
    a0 = a & ~(V - 1)
    if a + L <= n:
        return segment_pieces(a, a + L, a0, V, E)
    return segment_pieces(a, n, a0, V, E) + segment_pieces(0, a + L - n, (a0 - n) % (1 << 32), V, E)


@pytest.mark.parametrize("elem_bytes", [4, 2])
@pytest.mark.parametrize("dims", [(16, 8, 8), (128, 64, 64), (24, 16, 16), (20, 3, 7), (12, 4, 2), (8, 4, 3)])
def test_pipe_plan_in_bounds_aligned_and_covering(elem_bytes, dims):
    V = 16 // elem_bytes
    R = TILE + V
    n = dims[0] * dims[1] * dims[2]
    if n % V:
        pytest.skip("the pipelined kernel needs N % V == 0 (other grids take the per-thread kernel)")
    ntiles = (n + TILE - 1) // TILE
    rng = np.random.default_rng(n + elem_bytes)
    for trial in range(12):
        shifts = [0] * 27 if trial == 0 else [int(x) for x in rng.integers(0, n, 27)]
        if trial == 1:
            shifts = [n - 1 - (q % 5) for q in range(27)]  # runs that wrap in the last tile
        extra = sum(16 for s in shifts if s % V)
        for shift in shifts[:6]:
            covered = np.zeros(n, dtype=np.int32)
            for tile in range(ntiles):
                c0 = tile * TILE
                L = min(TILE, n - c0)
                assert L % V == 0
                a, a0, loads = loads_of(n, shift, c0, V)
                rem = shift % V
                assert a - a0 == rem  # the same for every tile of a launch
                loaded = np.zeros(R, dtype=bool)
                copied = 0
                for start, count, dst in loads:
                    assert count > 0 and start >= 0 and start + count <= n
                    assert (start * elem_bytes) % 16 == 0 and (count * elem_bytes) % 16 == 0
                    assert (dst * elem_bytes) % 16 == 0 and dst + count <= R
                    loaded[dst:dst + count] = True
                    copied += count * elem_bytes
                assert loaded[rem:rem + L].all()
                assert copied == L * elem_bytes + (16 if rem else 0)
                run = {(a + t) % n for t in range(L)}
                for g, cnt, s, kind in stores_of(n, shift, c0, V, elem_bytes):
                    nbytes = cnt * elem_bytes
                    assert 0 <= g and g + cnt <= n and s + cnt <= R
                    assert loaded[s:s + cnt].all()  # written back from loaded elements
                    assert all((g + i) in run for i in range(cnt))  # only the tile's own cells
                    if kind == "bulk":
                        assert (g * elem_bytes) % 16 == 0 and nbytes % 16 == 0 and (s * elem_bytes) % 16 == 0
                    else:
                        assert (g * elem_bytes) % nbytes == 0 and (s * elem_bytes) % nbytes == 0
                        assert (g * elem_bytes) % 16 == (s * elem_bytes) % 16
                    covered[g:g + cnt] += 1
            assert np.all(covered == 1)
        # the mbarrier's armed byte count (27 rows + markers) equals the bytes copied
        for tile in range(ntiles):
            c0 = tile * TILE
            L = min(TILE, n - c0)
            copied = sum(cnt * elem_bytes for s in shifts for _, cnt, _ in loads_of(n, s, c0, V)[2])
            assert copied == 27 * L * elem_bytes + extra
