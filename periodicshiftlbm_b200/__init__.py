"""B200-native (sm_100a) PeriodicShiftLBM lattice update.

The product is the CUDA library ``libpsl_b200.so`` (C ABI in include/psl.h); this package
is its host-side mirror of the reference's per-step API (see ``grid.py``) and the builder
(``build.py``).  Importing the package does not need a GPU; calling into it does.
"""
from .grid import (  # noqa: F401
    GridStruct,
    InfoStruct,
    SphereCase,
    applyBCPeriodicX,
    applyBCPeriodicY,
    applyCoarseFineGridCommunication,
    fillCoarseGridFromFine,
    applyLocalCellUpdate,
    applyStreaming,
    debug_cells,
    drag_coefficient,
    exportHistoryData,
    exportSectionCutPlot,
    sectionCut,
    fillEquilibriumFromFunction,
    getSphereDrag,
    getFlowReport,
    getForcingTorque,
    getSphereForce,
    getSphereForceAsync,
    getTorque,
    setBodyForce,
    setGivenRhoUxUyUz,
    setSmagorinskyConstant,
    setSphereCase,
    updateGrid,
)
from .cases import SphereConfig, config1, config2, make_sphere_grids  # noqa: F401

__version__ = "0.1.0"
