"""The C-ABI library loads, exports every entry point include/psl.h declares, validates
arguments, and fails loudly (no CPU fallback) without a GPU.  No GPU needed."""
import ctypes
import os
import re

import pytest

from periodicshiftlbm_b200 import _lib
from periodicshiftlbm_b200.cases import config1, config2

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "psl.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(psl_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), name
    # the binding covers the whole header
    assert set(names) <= set(_lib._SIGNATURES)


def test_version_string():
    assert b"sm_100a" in _lib.lib().psl_version()


def _info(nx, ny, nz):
    i = _lib.PslInfo()
    i.grid_id, i.res, i.nu, i.dt_phys = 0, 1.0, 0.01, 1.0
    i.cell_count_x, i.cell_count_y, i.cell_count_z = nx, ny, nz
    return i


@pytest.mark.parametrize("dims", [(0, 4, 4), (8, 1, 1), (2048, 2048, 1024)])
def test_invalid_grids_rejected_before_any_device_work(dims):
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.psl_grid_create(ctypes.byref(_info(*dims)), 0, ctypes.byref(h))
    assert rc == 1  # PSL_ERR_INVALID
    assert L.psl_last_error()
    assert not h.value


def test_unknown_storage_rejected():
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.psl_grid_create(ctypes.byref(_info(8, 8, 8)), 7, ctypes.byref(h)) == 1


def test_null_grid_arguments_rejected():
    L = _lib.lib()
    assert L.psl_apply_local_cell_update(None) == 1
    assert L.psl_apply_streaming(None) == 1
    assert L.psl_apply_coarse_fine_grid_communication(None, None) == 1
    assert L.psl_sphere_force_async(None, None, None) == 1
    assert L.psl_grid_get_layout(None, None, None) == 1
    assert L.psl_set_sgs_mlp_interval(None, 2) == 1
    assert b"null grid" in L.psl_last_error()


def test_unknown_grid_flags_rejected():
    """psl_grid_create_ex accepts PSL_GRID_ONE_MAPPING (1) only; anything else is refused
    before any device work."""
    L = _lib.lib()
    h = ctypes.c_void_p()
    for flags in (2, 4, 0x80000000):
        assert L.psl_grid_create_ex(ctypes.byref(_info(8, 8, 8)), 0, flags, ctypes.byref(h)) == 1
        assert b"flags" in L.psl_last_error()
        assert not h.value


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    from periodicshiftlbm_b200 import GridStruct, InfoStruct

    with pytest.raises(_lib.PslError):
        GridStruct(InfoStruct(cellCountX=8, cellCountY=8, cellCountZ=8, nu=0.01))


def test_update_counts_of_configurations():
    # config 1: every cell; config 2: the counts stated for the refined sphere case
    assert config1().updates_per_step() == 128 * 64 * 64
    c2 = config2()
    assert c2.updates_per_step() == 33554432 - 124 * 92 * 92 + 2 * 254 * 190 * 190 == 50843696
    assert c2.reference_updates_per_step() == 51315464
    fine = c2.infos()[1]
    assert (fine.cellCountX, fine.cellCountY, fine.cellCountZ) == (256, 192, 192)
    assert (fine.ox, fine.res) == (79.75, 0.5)
