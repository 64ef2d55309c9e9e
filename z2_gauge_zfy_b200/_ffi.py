"""ctypes binding of the C ABI declared in include/z2dqmc.h.

The shared library ``libz2dqmc.so`` is built in-tree (see ``build.py``).  There
is no fallback: if the library is missing or fails to load, importing the
compute entry points raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libz2dqmc.so")

Z2_NOBS_EQ = 7
Z2_NOBS_TAU = 7
Z2_NSTATS = 14

STATUS = {0: "Z2_OK", 1: "Z2_ERR_ARG", 2: "Z2_ERR_CUDA", 3: "Z2_ERR_NONFINITE",
          4: "Z2_ERR_STATE", 5: "Z2_ERR_NOMEM", 6: "Z2_ERR_TIMEOUT"}

# Every symbol include/z2dqmc.h declares.
EXPORTS = (
    "z2_create", "z2_destroy", "z2_last_error", "z2_chain_dims", "z2_set_config",
    "z2_get_config", "z2_pre", "z2_sweep", "z2_sweep_timed", "z2_get_green",
    "z2_get_obs_equal", "z2_get_obs_tau", "z2_get_stats", "z2_set_replay",
    "z2_get_decisions", "z2_logdet_grad", "z2_opk_mmult_R", "z2_opk_mmult_L",
    "z2_stab_UR", "z2_stab_UL", "z2_stab_green", "z2_stab_green_big",
    "z2_stab_green_noalloc", "z2_get_phase_cycles", "z2_tune_delay", "z2_get_obs_tau_k",
    "z2_sweep_global", "z2_get_global_stats", "z2_therm",
    # module-level mirrors on a chain's resident state
    "z2_propK_pre", "z2_propK_L", "z2_propK_R", "z2_propgrK_R", "z2_propT_pre", "z2_propT_L",
    "z2_propT_R", "z2_propgrT_R", "z2_wrap_pre", "z2_wrap_L", "z2_wrap_R", "z2_wrap_tau",
    "z2_dyn_reset", "z2_prop_slice_L", "z2_prop_slice_R", "z2_sweep_reset",
    "z2_obs_equal_calc", "z2_obs_equal_ave", "z2_obs_tau_calc", "z2_obs_tau_ave",
    "z2_get_prop", "z2_set_prop", "z2_get_propgr", "z2_tune", "z2_get_obs_equal_all",
)
# entry points (handle, chain, nt) and (handle, chain) of the state mirrors
STATE_NT = ("z2_propK_pre", "z2_propK_L", "z2_propK_R", "z2_propgrK_R", "z2_wrap_pre",
            "z2_wrap_tau", "z2_prop_slice_L", "z2_prop_slice_R", "z2_obs_equal_calc",
            "z2_obs_tau_calc")
STATE_CHAIN = ("z2_propT_pre", "z2_propT_L", "z2_propT_R", "z2_propgrT_R", "z2_dyn_reset")
Z2_NOALLOC_NMAX = 144


class Z2Error(RuntimeError):
    """A non-zero status returned by the library."""

    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class ChainParams(C.Structure):
    """``z2_chain_params``: the paramC_sets.txt fields of one chain."""
    _fields_ = [("RT", C.c_double), ("J", C.c_double), ("h", C.c_double),
                ("mu", C.c_double), ("Q", C.c_double),
                ("Nlx", C.c_int32), ("Nly", C.c_int32), ("Ltrot", C.c_int32),
                ("beta", C.c_double), ("Nwrap", C.c_int32), ("absolute", C.c_int32),
                ("seed", C.c_int32), ("rt_bond", C.POINTER(C.c_double))]


class Options(C.Structure):
    """``z2_options``."""
    _fields_ = [("delay_k", C.c_int32), ("record", C.c_int32), ("device", C.c_int32),
                ("tau", C.c_int32), ("graph", C.c_int32),
                ("delay_k_chain", C.POINTER(C.c_int32)),
                ("flush_shape_chain", C.POINTER(C.c_int32)), ("stab_exact", C.c_int32)]


_lib = None


def load():
    """Load the library (raises if it is absent: there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not built; run __graft_entry__.build() or "
                          "python -m z2_gauge_zfy_b200.build")
    lib = C.CDLL(LIB_PATH)
    vp, i32, dp = C.c_void_p, C.c_int32, C.POINTER(C.c_double)
    sig = {
        "z2_create": (C.c_int, [C.POINTER(vp), C.POINTER(ChainParams), i32, C.POINTER(Options)]),
        "z2_destroy": (C.c_int, [vp]),
        "z2_last_error": (C.c_char_p, [vp]),
        "z2_chain_dims": (C.c_int, [vp, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]),
        "z2_set_config": (C.c_int, [vp, i32, dp, i32]),
        "z2_get_config": (C.c_int, [vp, i32, dp, C.POINTER(i32)]),
        "z2_pre": (C.c_int, [vp]),
        "z2_sweep": (C.c_int, [vp, i32, i32]),
        "z2_sweep_timed": (C.c_int, [vp, i32, i32, C.POINTER(C.c_float)]),
        "z2_get_green": (C.c_int, [vp, i32, dp]),
        "z2_get_obs_equal": (C.c_int, [vp, i32, dp]),
        "z2_get_obs_tau": (C.c_int, [vp, i32, dp]),
        "z2_get_obs_tau_k": (C.c_int, [vp, i32, dp, dp]),
        "z2_get_stats": (C.c_int, [vp, i32, dp]),
        "z2_set_replay": (C.c_int, [vp, i32, dp, C.c_size_t]),
        "z2_get_decisions": (C.c_int, [vp, i32, C.POINTER(C.c_uint8), dp, C.c_size_t]),
        "z2_logdet_grad": (C.c_int, [vp, i32, dp, dp, dp]),
        "z2_opk_mmult_R": (C.c_int, [vp, i32, dp, i32, i32]),
        "z2_opk_mmult_L": (C.c_int, [vp, i32, dp, i32, i32]),
        "z2_stab_UR": (C.c_int, [vp, i32, dp, dp, dp]),
        "z2_stab_UL": (C.c_int, [vp, i32, dp, dp, dp]),
        "z2_stab_green": (C.c_int, [vp, i32, dp, dp, dp, dp, dp, dp, i32, dp]),
        "z2_stab_green_big": (C.c_int, [vp, i32, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp]),
        "z2_stab_green_noalloc": (C.c_int, [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp]),
        "z2_get_phase_cycles": (C.c_int, [vp, i32, dp]),
        "z2_sweep_global": (C.c_int, [vp, i32]),
        "z2_therm": (C.c_int, [vp, i32, dp]),
        "z2_get_global_stats": (C.c_int, [vp, i32, dp]),
        "z2_tune_delay": (C.c_int, [C.POINTER(ChainParams), i32, C.POINTER(Options),
                                   C.POINTER(i32)]),
        "z2_tune": (C.c_int, [C.POINTER(ChainParams), i32, C.POINTER(Options), C.POINTER(i32),
                             C.POINTER(i32)]),
        "z2_get_obs_equal_all": (C.c_int, [vp, dp]),
        "z2_wrap_L": (C.c_int, [vp, i32, i32, i32]),
        "z2_wrap_R": (C.c_int, [vp, i32, i32, i32]),
        "z2_sweep_reset": (C.c_int, [vp, i32, i32]),
        "z2_obs_equal_ave": (C.c_int, [vp, i32, i32]),
        "z2_obs_tau_ave": (C.c_int, [vp, i32, i32]),
        "z2_get_prop": (C.c_int, [vp, i32, dp, dp, dp, dp, dp, dp, dp]),
        "z2_set_prop": (C.c_int, [vp, i32, dp, dp, dp, dp, dp, dp, dp]),
        "z2_get_propgr": (C.c_int, [vp, i32, dp, dp, dp, dp]),
    }
    for name in STATE_NT:
        sig[name] = (C.c_int, [vp, i32, i32])
    for name in STATE_CHAIN:
        sig[name] = (C.c_int, [vp, i32])
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def dptr(a: np.ndarray):
    """Pointer to a C-contiguous float64 array."""
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def fmat(a) -> np.ndarray:
    """A column-major (Fortran-order) float64 matrix viewed as a flat C buffer."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)
