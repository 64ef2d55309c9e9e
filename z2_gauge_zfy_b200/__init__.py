"""B200-native (sm_100a, FP64) DQMC hot path for spinful fermions coupled to a
Z2 lattice gauge field -- a drop-in for the local-sweep path of
SONY932/z2_gauge_zfy (src/local_sweep.f90, src/multiply.f90,
src/stabilization.f90, src/dynamics.f90, src/obser_equal.f90,
src/obser_tau.f90).

The compute lives in the in-tree CUDA library ``libz2dqmc.so`` behind the C
ABI of ``include/z2dqmc.h``; this package is its host-side binding.
"""
from ._ffi import LIB_PATH, Z2Error, load  # noqa: F401
from .api import (FLUSH_SHAPES, OBS_EQ_NAMES, OBS_TAU_NAMES, STAT_NAMES,  # noqa: F401
                  Chain, Z2Batch, tune, tune_delay)

__all__ = ["Chain", "Z2Batch", "Z2Error", "load", "LIB_PATH", "OBS_EQ_NAMES",
           "OBS_TAU_NAMES", "STAT_NAMES", "tune", "tune_delay", "FLUSH_SHAPES"]
