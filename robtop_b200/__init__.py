"""robtop_b200 — B200-native (sm_100a) drop-in for robtop's multigrid solver hot path.

The compute lives in ``librtb200.so`` (hand-written CUDA for sm_100a behind the
C ABI of ``include/rtb200.h``).  This package is the host-side mirror of the
reference's interfaces:

* :mod:`robtop_b200.grid` — ``HierarchyGrid`` / ``Grid`` (grid/Grid.h)
* :mod:`robtop_b200.optimization` — the free functions of optimization/optimization.h
* :mod:`robtop_b200.configs` — seeded synthetic domains of the benchmark configurations
"""
from . import _capi  # noqa: F401
from ._capi import (FP32, FP64, FP64_FINE, LAYOUT_DENSE, LAYOUT_REF_GS, MODE_NSCF, MODE_NSFF, MODE_WSCF, MODE_WSFF,  # noqa: F401
                    SMOOTH_CHEBY, SMOOTH_GS, SMOOTH_JACOBI, SMOOTH_SGS, WORST_BLOCK_LANCZOS, WORST_LANCZOS, WORST_MODPM,
                    RTError, lib)
from .grid import Context, Grid, HierarchyGrid, default_params, pcg_batch, voxelize_mesh  # noqa: F401

__all__ = ["Context", "Grid", "HierarchyGrid", "default_params", "pcg_batch", "voxelize_mesh", "lib", "RTError"]
