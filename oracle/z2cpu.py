"""ctypes binding of the C restatement (oracle/c/z2cpu.c).  Test
infrastructure and CPU baseline only."""
import ctypes as C

import numpy as np

from . import build_cpu

_lib = None
_dp = C.POINTER(C.c_double)


def _load():
    global _lib
    if _lib is None:
        lib = C.CDLL(build_cpu.build())
        lib.z2cpu_run.restype = C.c_int
        lib.z2cpu_run.argtypes = [_dp, C.POINTER(C.c_int), _dp, _dp, C.POINTER(C.c_uint8), _dp, _dp]
        lib.z2cpu_new.restype = C.c_void_p
        lib.z2cpu_new.argtypes = [_dp, C.POINTER(C.c_int)]
        lib.z2cpu_pre.restype = None
        lib.z2cpu_pre.argtypes = [C.c_void_p]
        lib.z2cpu_bin.restype = C.c_double
        lib.z2cpu_bin.argtypes = [C.c_void_p, C.c_int, _dp, C.POINTER(C.c_uint8)]
        lib.z2cpu_state.restype = None
        lib.z2cpu_state.argtypes = [C.c_void_p, _dp, _dp, _dp]
        lib.z2cpu_free.restype = None
        lib.z2cpu_free.argtypes = [C.c_void_p]
        _lib = lib
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


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
    rc = lib.z2cpu_run(_d(dpar), ipar.ctypes.data_as(C.POINTER(C.c_int)), _d(obs), _d(G),
                       dec.ctypes.data_as(C.POINTER(C.c_uint8)) if record else None, _d(st),
                       C.byref(sec))
    if rc != 0:
        raise MemoryError("z2cpu_run: chain allocation failed")
    return dict(obs=obs, G=G.reshape(N, N).T.copy(),
                decisions=dec.reshape(2, Ltrot, 2 * N) if record else None,
                acc=st[0], Xmaxm=st[1], Xmeanm=st[2], iseed=int(st[3]), seconds=sec.value)


class CpuChain:
    """One chain of the C restatement kept resident between bins (the
    reference keeps its chain in process memory): seeded start, ``pre()``,
    then ``bin()`` per bin."""

    def __init__(self, RT, J, h, mu, beta, Nlx, Nly, Ltrot, Nwrap, seed, absolute=1):
        self.lib = _load()
        self.N, self.Ltrot = Nlx * Nly, Ltrot
        dpar = np.array([RT, J, h, mu, beta], dtype=np.float64)
        ipar = np.array([Nlx, Nly, Ltrot, Nwrap, absolute, seed], dtype=np.int32)
        self.h = self.lib.z2cpu_new(_d(dpar), ipar.ctypes.data_as(C.POINTER(C.c_int)))
        if not self.h:
            raise MemoryError("z2cpu_new: chain allocation failed")

    @classmethod
    def from_chain(cls, ch):
        """From an object with the fields of a chain's parameters (RT, J, h,
        mu, beta, Nlx, Nly, Ltrot, Nwrap, seed, absolute)."""
        return cls(ch.RT, ch.J, ch.h, ch.mu, ch.beta, ch.Nlx, ch.Nly, ch.Ltrot, ch.Nwrap,
                   ch.seed, ch.absolute)

    def pre(self):
        self.lib.z2cpu_pre(self.h)

    def bin(self, nsweep=1, record=False):
        """One bin; returns (seconds, obs[7], decisions [2, Ltrot, 2N] or None)."""
        obs = np.zeros(7)
        dec = np.zeros(2 * self.Ltrot * 2 * self.N, dtype=np.uint8) if record else None
        sec = self.lib.z2cpu_bin(self.h, nsweep, _d(obs),
                                 dec.ctypes.data_as(C.POINTER(C.c_uint8)) if record else None)
        return sec, obs, (dec.reshape(2, self.Ltrot, 2 * self.N) if record else None)

    def state(self):
        """dict(G, sigma [2N, Ltrot] (the Fortran array sigma(2N, Ltrot)), acc,
        Xmaxm, Xmeanm, iseed)."""
        N = self.N
        G = np.zeros(N * N)
        sig = np.zeros(2 * N * self.Ltrot)
        st = np.zeros(4)
        self.lib.z2cpu_state(self.h, _d(G), _d(sig), _d(st))
        return dict(G=G.reshape(N, N).T.copy(), sigma=sig.reshape(self.Ltrot, 2 * N).T.copy(),
                    acc=st[0], Xmaxm=st[1], Xmeanm=st[2], iseed=int(st[3]))

    def close(self):
        if self.h:
            self.lib.z2cpu_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
