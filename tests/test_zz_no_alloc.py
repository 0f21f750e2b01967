"""psl_momentum_exchange_force_noalloc: the force reduction for callers that cannot
allocate device memory (step loops inside CUDA stream capture, memory owned by another
allocator's pool or a fixed budget).  Its partial sums live in a fixed array inside the
library; the caller passes its own device buffers.  It must agree with the allocating
entry point, psl_sphere_force, on the same state -- call after call, since the fixed
array keeps the previous call's contents.

Collected last (file name) so a failure here does not hide the other tests' results."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 sums over the same cells, partitioned into different blocks


def _box(case, info):
    """The sphere's box exactly as psl_sphere_force computes it (float32 arithmetic,
    getSphereDrag's bounds, flowAroundSphereMainSingle.cu:105-110)."""
    f = np.float32
    lo, hi = [], []
    for c, o, n in zip(case.sphere, (info.ox, info.oy, info.oz), (info.cellCountX, info.cellCountY, info.cellCountZ)):
        a = int((f(c) - f(case.radius) - f(o)) / f(info.res))
        b = int((f(c) + f(case.radius) - f(o)) / f(info.res)) + 2
        lo.append(max(a, 0))
        hi.append(min(b, n))
    return np.array(lo, dtype=np.int32), np.array(hi, dtype=np.int32)


def _rows_with_shifts(f_logical, shifts, stride):
    """Lay out logical populations the way a periodic-shift grid stores them:
    row q holds population q of cell c at (c + shift_q) mod N."""
    n = f_logical.shape[1]
    rows = np.zeros((27, stride), dtype=np.float32)
    cells = np.arange(n)
    for q in range(27):
        rows[q, (cells + shifts[q]) % n] = f_logical[q]
    return rows


def test_noalloc_force_matches_allocating_entry_point():
    import torch

    from periodicshiftlbm_b200 import _lib, getSphereForce, updateGrid
    from periodicshiftlbm_b200.cases import SphereConfig, make_sphere_grids

    cfg = SphereConfig(name="noalloc", nx=48, ny=24, nz=24, sphere=(14.0, 12.0, 12.0), radius=4.0, u_in=0.05,
                       nu=0.01, smagorinsky=0.1)
    grids, case = make_sphere_grids(cfg)
    g = grids[0]
    info = g.Info
    n = info.cellCount
    lo, hi = _box(case, info)
    L = _lib.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(5)
    for call in range(2):  # two calls in a row: the fixed array keeps the previous contents
        for _ in range(7 + 5 * call):
            updateGrid(grids, 0)
        want = getSphereForce(g, case)  # the allocating entry point
        # the caller's own device buffers (allocated by the caller, not by the library)
        shifts = (g.shifter if call == 0 else rng.integers(0, n, 27)).astype(np.int32)
        stride = n + 96
        rows = torch.from_numpy(_rows_with_shifts(g.fArray, shifts, stride)).cuda()
        markers = torch.from_numpy(g.markers).cuda()
        out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = L.psl_momentum_exchange_force_noalloc(
            ctypes.c_void_p(rows.data_ptr()), stride, shifts.ctypes.data, n, ctypes.c_void_p(markers.data_ptr()),
            info.cellCountX, info.cellCountY, info.cellCountZ, lo.ctypes.data, hi.ctypes.data,
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.psl_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.allclose(got, want, rtol=TOL, atol=TOL * np.abs(want).max()), (call, got, want)
        assert abs(want[0]) > 0


def test_noalloc_force_rejects_boxes_beyond_its_fixed_scratch():
    import torch

    from periodicshiftlbm_b200 import _lib

    L = _lib.lib()
    nx = ny = nz = 168  # 4,741,632 cells > 4,194,304
    n = nx * ny * nz
    rows = torch.zeros(27, n, dtype=torch.float32, device="cuda")
    markers = torch.zeros(n, dtype=torch.uint8, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    shifts = np.zeros(27, dtype=np.int32)
    lo = np.zeros(3, dtype=np.int32)
    hi = np.array([nx, ny, nz], dtype=np.int32)
    rc = L.psl_momentum_exchange_force_noalloc(
        ctypes.c_void_p(rows.data_ptr()), n, shifts.ctypes.data, n, ctypes.c_void_p(markers.data_ptr()), nx, ny, nz,
        lo.ctypes.data, hi.ctypes.data, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"4194304" in L.psl_last_error()


def test_noalloc_force_in_a_captured_graph_and_after_a_larger_box():
    """One call outside capture, then a call captured into a CUDA graph (stream capture
    fails on any allocation or synchronisation) and replayed; and a call over the whole grid
    before the sphere's box, so the fixed partial sums hold more blocks than the second call
    writes.  Both give psl_sphere_force's result."""
    import torch

    from periodicshiftlbm_b200 import _lib, getSphereForce, updateGrid
    from periodicshiftlbm_b200.cases import SphereConfig, make_sphere_grids

    cfg = SphereConfig(name="noalloc", nx=48, ny=24, nz=24, sphere=(14.0, 12.0, 12.0), radius=4.0, u_in=0.05,
                       nu=0.01, smagorinsky=0.1)
    grids, case = make_sphere_grids(cfg)
    g = grids[0]
    info = g.Info
    n = info.cellCount
    for _ in range(9):
        updateGrid(grids, 0)
    want = getSphereForce(g, case)
    lo, hi = _box(case, info)
    whole_lo = np.zeros(3, dtype=np.int32)
    whole_hi = np.array([info.cellCountX, info.cellCountY, info.cellCountZ], dtype=np.int32)
    L = _lib.lib()
    shifts = g.shifter.astype(np.int32)
    rows = torch.from_numpy(_rows_with_shifts(g.fArray, shifts, n)).cuda()
    markers = torch.from_numpy(g.markers).cuda()
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    whole = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()

    def call(box_lo, box_hi, dst):
        return L.psl_momentum_exchange_force_noalloc(
            ctypes.c_void_p(rows.data_ptr()), n, shifts.ctypes.data, n, ctypes.c_void_p(markers.data_ptr()),
            info.cellCountX, info.cellCountY, info.cellCountZ, box_lo.ctypes.data, box_hi.ctypes.data,
            ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(s.cuda_stream))

    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        assert call(whole_lo, whole_hi, whole) == 0, L.psl_last_error()  # outside capture, larger box
        assert call(lo, hi, out) == 0, L.psl_last_error()                # then the sphere's box
    torch.cuda.synchronize()
    assert np.allclose(out.cpu().numpy(), want, rtol=TOL, atol=TOL * np.abs(want).max())
    out.fill_(float("nan"))
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        assert call(lo, hi, out) == 0, L.psl_last_error()
    torch.cuda.synchronize()
    graph.replay()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.allclose(got, want, rtol=TOL, atol=TOL * np.abs(want).max()), (got, want)
    assert np.all(np.isfinite(whole.cpu().numpy()))
    del graph
    for gr in grids:
        gr.close()


def test_noalloc_force_over_more_blocks_than_one_staged_chunk():
    """A box of more than 512 x 4096 cells: the final sum then stages the partial sums in
    two chunks of shared memory.  The sphere sits against the top of the grid, so solid
    cells fall into blocks of the second chunk; the whole grid's force equals the force over
    the sphere's own box (one chunk), since only solid cells contribute."""
    import torch

    from periodicshiftlbm_b200 import _lib, updateGrid
    from periodicshiftlbm_b200.cases import SphereConfig, make_sphere_grids

    cfg = SphereConfig(name="noalloc_big", nx=132, ny=128, nz=128, sphere=(60.0, 64.0, 121.5), radius=6.0,
                       u_in=0.05, nu=0.01, smagorinsky=0.1)
    grids, case = make_sphere_grids(cfg)
    g = grids[0]
    info = g.Info
    n = info.cellCount
    assert n > 512 * 4096
    for _ in range(3):
        updateGrid(grids, 0)
    lo, hi = _box(case, info)
    whole_lo = np.zeros(3, dtype=np.int32)
    whole_hi = np.array([info.cellCountX, info.cellCountY, info.cellCountZ], dtype=np.int32)
    markers_host = g.markers
    solid = (markers_host.reshape(-1) & 7) == 2
    ks = np.nonzero(solid)[0] // (info.cellCountX * info.cellCountY)
    assert ks.max() >= 125  # solid cells in blocks 512 and above of the whole-grid box
    L = _lib.lib()
    shifts = g.shifter.astype(np.int32)
    rows = torch.from_numpy(_rows_with_shifts(g.fArray, shifts, n)).cuda()
    markers = torch.from_numpy(markers_host).cuda()
    whole = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    box = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()

    def call(box_lo, box_hi, dst):
        return L.psl_momentum_exchange_force_noalloc(
            ctypes.c_void_p(rows.data_ptr()), n, shifts.ctypes.data, n, ctypes.c_void_p(markers.data_ptr()),
            info.cellCountX, info.cellCountY, info.cellCountZ, box_lo.ctypes.data, box_hi.ctypes.data,
            ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(s.cuda_stream))

    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        assert call(whole_lo, whole_hi, whole) == 0, L.psl_last_error()
        assert call(lo, hi, box) == 0, L.psl_last_error()
    torch.cuda.synchronize()
    w, b = whole.cpu().numpy(), box.cpu().numpy()
    assert np.all(np.isfinite(w)) and abs(b).max() > 0
    assert np.allclose(w, b, rtol=TOL, atol=TOL * np.abs(b).max()), (w, b)
    for gr in grids:
        gr.close()
