"""suli_b200 — B200 (sm_100a) implementation of the SuLi-IC per-time-step hot path.

The CUDA kernels and the C-ABI live in csrc/ and build into lib/libsuli_gpu.so; this
package is the host-side mirror of the reference's subroutine surface (solver.Solver) and
the synthetic cases (cases).  Load it by path, e.g.

    import importlib.util, sys
    spec = importlib.util.spec_from_file_location(
        "suli_b200", "suli-openmp_b200/__init__.py",
        submodule_search_locations=["suli-openmp_b200"])
"""
from ._abi import (FIELD, FIELD_NAMES, SCALAR, SuliParams, SuliStepStats, default_params,
                   field_extent, field_shape, load_library, LIB_PATH)
from .solver import Solver, SuliError
from . import cases, fileio, learned, mms_weng, snapshots

__all__ = [
    "FIELD", "FIELD_NAMES", "SCALAR", "SuliParams", "SuliStepStats", "default_params",
    "field_extent", "field_shape", "load_library", "LIB_PATH", "Solver", "SuliError", "cases", "fileio",
    "learned", "mms_weng", "snapshots",
]
