"""ctypes binding of the C restatement (oracle/c/z2cpu.c).  Test
infrastructure and CPU baseline only."""
import ctypes as C

import numpy as np

from . import build_cpu

_lib = None


def _load():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build_cpu.build())
        _lib.z2cpu_run.restype = C.c_int
        dp = C.POINTER(C.c_double)
        _lib.z2cpu_run.argtypes = [dp, C.POINTER(C.c_int), dp, dp, C.POINTER(C.c_uint8), dp, dp]
    return _lib


def run(RT, J, h, mu, beta, Nlx, Nly, Ltrot, Nwrap, seed, nbins=1, nsweep=1, absolute=1,
        record=False):
    """Returns dict(obs [nbins, 7], G, decisions [2, Ltrot, 2N] or None, acc,
    Xmaxm, Xmeanm, iseed, seconds)."""
    lib = _load()
    N = Nlx * Nly
    dpar = np.array([RT, J, h, mu, beta], dtype=np.float64)
    ipar = np.array([Nlx, Nly, Ltrot, Nwrap, absolute, seed, nbins, nsweep], dtype=np.int32)
    obs = np.zeros((nbins, 7))
    G = np.zeros(N * N)
    dec = np.zeros(2 * Ltrot * 2 * N, dtype=np.uint8) if record else None
    st = np.zeros(4)
    sec = C.c_double()
    dptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    lib.z2cpu_run(dptr(dpar), ipar.ctypes.data_as(C.POINTER(C.c_int)), dptr(obs), dptr(G),
                  dec.ctypes.data_as(C.POINTER(C.c_uint8)) if record else None, dptr(st),
                  C.byref(sec))
    return dict(obs=obs, G=G.reshape(N, N).T.copy(),
                decisions=dec.reshape(2, Ltrot, 2 * N) if record else None,
                acc=st[0], Xmaxm=st[1], Xmeanm=st[2], iseed=int(st[3]), seconds=sec.value)
