"""The header-only C++ mirror (include/psl.hpp) and the reference-style example driver
(examples/flow_around_sphere.cpp): they compile against the library (no GPU needed), and
on a GPU the example's drag equals the Python API's on the same case and steps."""
import os
import re
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(REPO, "tests", "_build")
LIBDIR = os.path.join(REPO, "periodicshiftlbm_b200")
EXE = os.path.join(BUILD, "flow_around_sphere")


def _gxx():
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if not gxx:
        pytest.skip("no host C++ compiler")
    return gxx


def build_example():
    os.makedirs(BUILD, exist_ok=True)
    lib = os.path.join(LIBDIR, "libpsl_b200.so")
    if not os.path.exists(lib):
        pytest.skip("libpsl_b200.so not built")
    subprocess.run([_gxx(), "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "examples", "flow_around_sphere.cpp"), lib, f"-Wl,-rpath,{LIBDIR}", "-o", EXE],
                   check=True)
    return EXE


def test_mirror_and_example_compile_and_link():
    assert os.path.exists(build_example())


@pytest.mark.gpu
@pytest.mark.parametrize("sponge", [False, True])
def test_example_drag_equals_python_api(sponge):
    """Also with the C++ per-cell getSmagorinskyConstant hook against the same hook in
    Python (cases.sponge_smagorinsky, SphereConfig.cs_mode = 1)."""
    from periodicshiftlbm_b200 import getSphereDrag, updateGrid
    from periodicshiftlbm_b200.cases import config2, make_sphere_grids

    scale, steps = 0.125, 12
    cmd = [build_example(), str(steps), str(scale)] + (["sponge"] if sponge else [])
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    drag_cpp = float(re.search(r"drag (\S+)", out).group(1))
    grids, case = make_sphere_grids(config2(scale=scale, cs_mode=1 if sponge else 0))
    for _ in range(steps):
        updateGrid(grids, 0)
    drag_py = getSphereDrag(grids[1], case)
    for g in grids:
        g.close()
    assert drag_cpp == pytest.approx(drag_py, rel=1e-12, abs=0.0), (drag_cpp, drag_py)
