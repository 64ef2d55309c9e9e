"""Host-side mirror of the reference's module interfaces for the DQMC hot path.

``Z2Batch`` owns a batch of independent Markov chains on one GPU (the
reference runs one chain per MPI rank).  Its methods mirror
``LocalSweep%pre`` / ``%sweep`` (src/local_sweep.f90:87-195), the readback of
``ObserEqual`` / ``ObserTau`` (src/obser_equal.f90, src/obser_tau.f90) and the
drift statistics of ``Propagator`` / ``PropGreen`` (src/process_matrix.f90).
The module-level functions mirror ``OperatorKin%mmult_R/L``
(src/operator_kin.f90:61-145) and the ``stab_*`` routines of
src/stabilization.f90 on single matrices.

Matrices are numpy arrays in natural (row, column) indexing; they are
converted to the library's column-major layout at the boundary.  Errors raise
``Z2Error`` (the reference would print and ``stop``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from ._ffi import ChainParams, Options, Z2Error, dptr, fmat

OBS_EQ_NAMES = ("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_shift", "cdw_ratio",
                "density")
OBS_TAU_NAMES = ("spin", "single", "pair_d", "pair_s", "charge_d", "charge_s", "curxx")
PHASE_NAMES = ("kin", "propose", "flush", "obs_equal", "wrap_stab", "dyn", "stab_U", "stab_green",
               "eval", "cols", "pending", "stack")
STAT_NAMES = ("acc", "Xmaxm", "Xmeanm", "Xmaxm_tau0", "Xmaxm_tau1", "Xmaxm_tau2",
              "Xmeanm_tau0", "Xmeanm_tau1", "Xmeanm_tau2", "accepted", "proposed", "draws",
              "nobs", "nobst")


@dataclass
class Chain:
    """Parameters of one chain: the hot-path lines of paramC_sets.txt
    (src/calc_basic.f90:52-62) and this chain's row of seeds.txt."""
    RT: float = 1.0
    J: float = 0.5
    h: float = 0.5
    mu: float = 0.0
    Q: float = 1.0
    Nlx: int = 4
    Nly: int = 4
    Ltrot: int = 40
    beta: float = 4.0
    Nwrap: int = 10
    absolute: int = 1
    seed: int = 12345
    rt_bond: np.ndarray | None = None

    @property
    def N(self):
        return self.Nlx * self.Nly


def _check(lib, h, code):
    if code != 0:
        msg = lib.z2_last_error(h)
        raise Z2Error(code, msg.decode() if msg else "")


def integrate_susc(gk: np.ndarray, dtau: float) -> np.ndarray:
    """Static susceptibility per momentum, dtau * sum_tau gk(k, tau)
    (m_integrate_susc_2_mom, src/fourier_trans.f90:165-177)."""
    return gk.sum(axis=1) * dtau


def integrate_susc_freq(gk: np.ndarray, dtau: float) -> np.ndarray:
    """Matsubara transform of the k = 0 row, dtau * sum_tau
    exp(2 pi i (tau-1)(w-1)/Ltrot) gk(0, tau), w = 1..Ltrot
    (m_integrate_susc_2_freq, src/fourier_trans.f90:179-191)."""
    L = gk.shape[1]
    t = np.arange(L)
    ph = np.exp(2j * np.pi * np.outer(t, t) / L)
    return (ph @ gk[0]) * dtau


def _params(chains):
    """ctypes array of z2_chain_params (and the per-bond arrays it points to)."""
    n = len(chains)
    arr = (ChainParams * n)()
    keep = []
    for i, ch in enumerate(chains):
        p = arr[i]
        p.RT, p.J, p.h, p.mu, p.Q = ch.RT, ch.J, ch.h, ch.mu, ch.Q
        p.Nlx, p.Nly, p.Ltrot, p.beta = ch.Nlx, ch.Nly, ch.Ltrot, ch.beta
        p.Nwrap, p.absolute, p.seed = ch.Nwrap, ch.absolute, ch.seed
        if ch.rt_bond is not None:
            rb = np.ascontiguousarray(ch.rt_bond, dtype=np.float64)
            if rb.shape != (2 * ch.N,):
                raise Z2Error(1, f"chain {i}: rt_bond has shape {rb.shape}, "
                                 f"needs one hopping per bond ({2 * ch.N},)")
            keep.append(rb)
            p.rt_bond = dptr(rb)
        else:
            p.rt_bond = None
    return arr, keep


def tune_delay(chains, device: int = 0, stab_exact: bool = False) -> np.ndarray:
    """Per-chain delayed-update rank picked by the library's autotuner
    (``z2_tune_delay``: short probe chains of each lattice size, timed at
    every candidate rank on the GPU)."""
    lib = _ffi.load()
    chains = list(chains)
    arr, _keep = _params(chains)
    opt = Options(0, 0, device, 0, 0, None, None, 1 if stab_exact else 0)
    k = np.zeros(len(chains), dtype=np.int32)
    code = lib.z2_tune_delay(arr, len(chains), C.byref(opt),
                             k.ctypes.data_as(C.POINTER(C.c_int32)))
    if code != 0:
        raise Z2Error(code, "z2_tune_delay failed")
    return k


FLUSH_SHAPES = {0: "by divisibility", 1: "bounded 16x16", 2: "bounded 8x8", 3: "8x8 blocks",
                4: "16x16 blocks", 5: "24x24 blocks", 6: "16x8 blocks", 7: "24x16 blocks"}


def tune(chains, device: int = 0, stab_exact: bool = False):
    """Per-chain delayed-update rank and flush tile shape picked jointly by the
    library's autotuner (``z2_tune``): returns (k, shape), int32 arrays."""
    lib = _ffi.load()
    chains = list(chains)
    arr, _keep = _params(chains)
    opt = Options(0, 0, device, 0, 0, None, None, 1 if stab_exact else 0)
    k = np.zeros(len(chains), dtype=np.int32)
    sh = np.zeros(len(chains), dtype=np.int32)
    code = lib.z2_tune(arr, len(chains), C.byref(opt), k.ctypes.data_as(C.POINTER(C.c_int32)),
                       sh.ctypes.data_as(C.POINTER(C.c_int32)))
    if code != 0:
        raise Z2Error(code, "z2_tune failed")
    return k, sh


class Z2Batch:
    """A batch of chains resident on one GPU (``z2_create``)."""

    def __init__(self, chains, delay_k=0, record: bool = False, device: int = 0,
                 tau: bool = False, graph: bool = False, delay_k_chain=None,
                 stab_exact: bool = False, flush_shape_chain=None):
        """delay_k: rank of the delayed updates for every chain (0 = built-in
        default per lattice size), or "auto" to run the autotuner
        (``z2_tune``) and use its per-chain ranks and flush tile shapes.
        stab_exact: stabilize with the reference's column-pivoted QR instead of
        the pre-pivoted QR (``z2_options.stab_exact``).  flush_shape_chain:
        per-chain tile shape of the rank-2k flush (``FLUSH_SHAPES``)."""
        self.lib = _ffi.load()
        self.chains = list(chains)
        n = len(self.chains)
        arr, self._rt_keep = _params(self.chains)
        if delay_k == "auto":
            delay_k_chain, flush_shape_chain = tune(self.chains, device, stab_exact)
            delay_k = 0
        self._kc = None
        kc_ptr = None
        if delay_k_chain is not None:
            self._kc = np.ascontiguousarray(delay_k_chain, dtype=np.int32)
            if self._kc.shape != (n,):
                raise Z2Error(1, f"delay_k_chain has shape {self._kc.shape}, "
                                 f"needs one rank per chain ({n},)")
            kc_ptr = self._kc.ctypes.data_as(C.POINTER(C.c_int32))
        self._fs = None
        fs_ptr = None
        if flush_shape_chain is not None:
            self._fs = np.ascontiguousarray(flush_shape_chain, dtype=np.int32)
            if self._fs.shape != (n,):
                raise Z2Error(1, f"flush_shape_chain has shape {self._fs.shape}, "
                                 f"needs one shape per chain ({n},)")
            fs_ptr = self._fs.ctypes.data_as(C.POINTER(C.c_int32))
        opt = Options(delay_k, 1 if record else 0, device, 1 if tau else 0, 1 if graph else 0,
                      kc_ptr, fs_ptr, 1 if stab_exact else 0)
        h = C.c_void_p()
        code = self.lib.z2_create(C.byref(h), arr, n, C.byref(opt))
        self.h = h
        if code != 0:
            msg = self.lib.z2_last_error(h)
            self.lib.z2_destroy(h)
            self.h = None
            raise Z2Error(code, msg.decode() if msg else "")

    # -- life cycle ---------------------------------------------------------
    def close(self):
        if self.h is not None:
            self.lib.z2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, code):
        _check(self.lib, self.h, code)

    # -- LocalSweep ----------------------------------------------------------
    def pre(self):
        """``Local_sweep_pre`` on every chain."""
        self._c(self.lib.z2_pre(self.h))

    def sweep(self, nsweep: int = 1, toggle: bool = False) -> None:
        """``Local_sweep`` (one bin of ``nsweep`` L+R sweep pairs) on every chain."""
        self._c(self.lib.z2_sweep(self.h, nsweep, 1 if toggle else 0))

    def sweep_timed(self, nsweep: int = 1, toggle: bool = False) -> float:
        """Like ``sweep``; returns the device time of the launch in ms."""
        ms = C.c_float()
        self._c(self.lib.z2_sweep_timed(self.h, nsweep, 1 if toggle else 0, C.byref(ms)))
        return float(ms.value)

    # -- configuration -------------------------------------------------------
    def _shaped(self, chain: int, name: str, a, shape: tuple) -> np.ndarray:
        """``a`` as float64 if it has ``shape`` (the library copies exactly
        that many values for this chain), else an argument error."""
        a = np.asarray(a, dtype=np.float64)
        if a.shape != shape:
            raise Z2Error(1, f"{name}: shape {a.shape}, chain {chain} needs {shape}")
        return a

    def _mats(self, chain: int, **arrays) -> list:
        """N x N matrices and length-N vectors (names starting with D) of one
        chain, checked and in the library's layout."""
        N = self.dims(chain)[0]
        out = []
        for name, a in arrays.items():
            if name.startswith("D"):
                out.append(np.ascontiguousarray(self._shaped(chain, name, a, (N,))))
            else:
                out.append(fmat(self._shaped(chain, name, a, (N, N))).ravel())
        return out

    def dims(self, chain: int):
        N, L, S = C.c_int32(), C.c_int32(), C.c_int32()
        self._c(self.lib.z2_chain_dims(self.h, chain, C.byref(N), C.byref(L), C.byref(S)))
        return N.value, L.value, S.value

    def get_config(self, chain: int):
        """sigma(2N, Ltrot) and the ranf state (``conf_out``)."""
        N, L, _ = self.dims(chain)
        buf = np.empty(2 * N * L)
        seed = C.c_int32()
        self._c(self.lib.z2_get_config(self.h, chain, dptr(buf), C.byref(seed)))
        return buf.reshape(L, 2 * N).T.copy(), seed.value

    def set_config(self, chain: int, sigma, iseed: int):
        """Load sigma(2N, Ltrot) and the ranf state (``conf_in``)."""
        N, L, _ = self.dims(chain)
        s = fmat(self._shaped(chain, "sigma", sigma, (2 * N, L))).ravel()
        self._c(self.lib.z2_set_config(self.h, chain, dptr(s), int(iseed)))

    # -- readback ------------------------------------------------------------
    def green(self, chain: int) -> np.ndarray:
        N = self.dims(chain)[0]
        buf = np.empty(N * N)
        self._c(self.lib.z2_get_green(self.h, chain, dptr(buf)))
        return buf.reshape(N, N).T.copy()

    def obs_equal(self, chain: int) -> dict:
        buf = np.empty(_ffi.Z2_NOBS_EQ)
        self._c(self.lib.z2_get_obs_equal(self.h, chain, dptr(buf)))
        return dict(zip(OBS_EQ_NAMES, buf.tolist()))

    def obs_equal_all(self) -> np.ndarray:
        """Bin observables of every chain, [n_chains, 7] in the order of
        ``OBS_EQ_NAMES`` (``z2_get_obs_equal_all``: one gather, one copy)."""
        buf = np.empty((len(self.chains), _ffi.Z2_NOBS_EQ))
        self._c(self.lib.z2_get_obs_equal_all(self.h, dptr(buf)))
        return buf

    def obs_tau(self, chain: int) -> dict:
        N, L, _ = self.dims(chain)
        buf = np.empty(7 * N * L)
        self._c(self.lib.z2_get_obs_tau(self.h, chain, dptr(buf)))
        a = buf.reshape(7, L, N)
        return {k: a[q].T.copy() for q, k in enumerate(OBS_TAU_NAMES)}

    def obs_tau_k(self, chain: int) -> dict:
        """Time-displaced correlators in momentum space (``z2_get_obs_tau_k``,
        Fourier_R_to_K of the reference's output layer): name -> complex
        array [N (momentum index), Ltrot]."""
        N, L, _ = self.dims(chain)
        re = np.empty(7 * N * L)
        im = np.empty(7 * N * L)
        self._c(self.lib.z2_get_obs_tau_k(self.h, chain, dptr(re), dptr(im)))
        a = (re + 1j * im).reshape(7, L, N)
        return {k: a[q].T.copy() for q, k in enumerate(OBS_TAU_NAMES)}

    def therm(self, nwarm: int) -> np.ndarray:
        """Boson-only warm-up of every chain (``z2_therm``); returns each
        chain's mean accepted fraction.  Call before ``pre``."""
        acc = np.empty(len(self.chains))
        self._c(self.lib.z2_therm(self.h, nwarm, dptr(acc)))
        return acc

    def sweep_global(self, nglobal: int):
        """Global Wolff-in-tau moves of every chain (``z2_sweep_global``,
        Sweep_global%sweep of the reference)."""
        self._c(self.lib.z2_sweep_global(self.h, nglobal))

    def global_stats(self, chain: int) -> dict:
        buf = np.empty(5)
        self._c(self.lib.z2_get_global_stats(self.h, chain, dptr(buf)))
        return dict(zip(("acc", "size_cluster", "accepted", "proposed", "is_beta"), buf.tolist()))

    def stats(self, chain: int) -> dict:
        buf = np.empty(_ffi.Z2_NSTATS)
        self._c(self.lib.z2_get_stats(self.h, chain, dptr(buf)))
        return dict(zip(STAT_NAMES, buf.tolist()))

    def phase_cycles(self, chain: int) -> dict:
        """SM cycles per phase accumulated since creation (tracing)."""
        buf = np.empty(len(PHASE_NAMES))
        self._c(self.lib.z2_get_phase_cycles(self.h, chain, dptr(buf)))
        return dict(zip(PHASE_NAMES, buf.tolist()))

    def set_replay(self, chain: int, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._c(self.lib.z2_set_replay(self.h, chain, dptr(v) if v.size else None, v.size))

    def decisions(self, chain: int):
        """Decisions and ratios of the last half-sweeps as arrays [2, Ltrot, 2N]
        (L half-sweep then R)."""
        N, L, _ = self.dims(chain)
        n = 2 * L * 2 * N
        dec = np.empty(n, dtype=np.uint8)
        rat = np.empty(n)
        self._c(self.lib.z2_get_decisions(self.h, chain, dec.ctypes.data_as(C.POINTER(C.c_uint8)),
                                          dptr(rat), n))
        return dec.reshape(2, L, 2 * N), rat.reshape(2, L, 2 * N)

    def logdet_grad(self, chain: int):
        """log|det(1+B)| of one spin sector, d/dt_b (2N) and d/dmu."""
        N = self.dims(chain)[0]
        ld, dmu = C.c_double(), C.c_double()
        g = np.empty(2 * N)
        self._c(self.lib.z2_logdet_grad(self.h, chain, C.byref(ld), dptr(g), C.byref(dmu)))
        return ld.value, g, dmu.value

    # -- module-level mirrors --------------------------------------------------
    def opk_mmult_R(self, chain: int, M, nt: int, nflag: int) -> np.ndarray:
        """B_nt^nflag M (``OperatorKin%mmult_R``), nt = 1..Ltrot."""
        (b,) = self._mats(chain, M=M)
        self._c(self.lib.z2_opk_mmult_R(self.h, chain, dptr(b), nt, nflag))
        n = int(round(np.sqrt(b.size)))
        return b.reshape(n, n).T.copy()

    def opk_mmult_L(self, chain: int, M, nt: int, nflag: int) -> np.ndarray:
        """M B_nt^nflag (``OperatorKin%mmult_L``)."""
        (b,) = self._mats(chain, M=M)
        self._c(self.lib.z2_opk_mmult_L(self.h, chain, dptr(b), nt, nflag))
        n = int(round(np.sqrt(b.size)))
        return b.reshape(n, n).T.copy()

    def _stab_u(self, fn, chain, U, D, V):
        u, d, v = self._mats(chain, U=U, D=D, V=V)
        n = d.size
        d = d.copy()
        self._c(fn(self.h, chain, dptr(u), dptr(d), dptr(v)))
        return u.reshape(n, n).T.copy(), d, v.reshape(n, n).T.copy()

    def stab_UR(self, chain, U, D, V):
        """``stab_UR``: returns the new (UR, DR, VR)."""
        return self._stab_u(self.lib.z2_stab_UR, chain, U, D, V)

    def stab_UL(self, chain, U, D, V):
        """``stab_UL``: returns the new (UL, DL, VL)."""
        return self._stab_u(self.lib.z2_stab_UL, chain, U, D, V)

    def stab_green(self, chain, UR, DR, VR, UL, DL, VL, nt: int) -> np.ndarray:
        args = self._mats(chain, UR=UR, DR=DR, VR=VR, UL=UL, DL=DL, VL=VL)
        n = args[1].size
        g = np.empty(n * n)
        self._c(self.lib.z2_stab_green(self.h, chain, *[dptr(a) for a in args], nt, dptr(g)))
        return g.reshape(n, n).T.copy()

    def stab_green_big(self, chain, UR, DR, VR, UL, DL, VL):
        args = self._mats(chain, UR=UR, DR=DR, VR=VR, UL=UL, DL=DL, VL=VL)
        n = args[1].size
        outs = [np.empty(n * n) for _ in range(4)]
        self._c(self.lib.z2_stab_green_big(self.h, chain, *[dptr(a) for a in args],
                                           *[dptr(o) for o in outs]))
        return tuple(o.reshape(n, n).T.copy() for o in outs)

    # -- module-level mirrors on a chain's resident state -----------------------
    # (src/multiply.f90, src/stabilization.f90:374-514, src/dynamics.f90:41-48,
    # src/localK.f90:347-398, src/local_sweep.f90:56-71, src/obser_equal.f90,
    # src/obser_tau.f90); nt follows the reference (1..Ltrot, wraps 0..Ltrot)
    def propK_pre(self, chain: int, nt: int):
        self._c(self.lib.z2_propK_pre(self.h, chain, nt))

    def propK_L(self, chain: int, nt: int):
        self._c(self.lib.z2_propK_L(self.h, chain, nt))

    def propK_R(self, chain: int, nt: int):
        self._c(self.lib.z2_propK_R(self.h, chain, nt))

    def propgrK_R(self, chain: int, nt: int):
        self._c(self.lib.z2_propgrK_R(self.h, chain, nt))

    def propT_pre(self, chain: int):
        self._c(self.lib.z2_propT_pre(self.h, chain))

    def propT_L(self, chain: int):
        self._c(self.lib.z2_propT_L(self.h, chain))

    def propT_R(self, chain: int):
        self._c(self.lib.z2_propT_R(self.h, chain))

    def propgrT_R(self, chain: int):
        self._c(self.lib.z2_propgrT_R(self.h, chain))

    def wrap_pre(self, chain: int, nt: int):
        self._c(self.lib.z2_wrap_pre(self.h, chain, nt))

    def wrap_L(self, chain: int, nt: int, flag: bool = True):
        self._c(self.lib.z2_wrap_L(self.h, chain, nt, 1 if flag else 0))

    def wrap_R(self, chain: int, nt: int, flag: bool = True):
        self._c(self.lib.z2_wrap_R(self.h, chain, nt, 1 if flag else 0))

    def wrap_tau(self, chain: int, nt: int):
        self._c(self.lib.z2_wrap_tau(self.h, chain, nt))

    def dyn_reset(self, chain: int):
        self._c(self.lib.z2_dyn_reset(self.h, chain))

    def prop_slice_L(self, chain: int, nt: int):
        self._c(self.lib.z2_prop_slice_L(self.h, chain, nt))

    def prop_slice_R(self, chain: int, nt: int):
        self._c(self.lib.z2_prop_slice_R(self.h, chain, nt))

    def sweep_reset(self, chain: int, toggle: bool = False):
        self._c(self.lib.z2_sweep_reset(self.h, chain, 1 if toggle else 0))

    def obs_equal_calc(self, chain: int, nt: int):
        self._c(self.lib.z2_obs_equal_calc(self.h, chain, nt))

    def obs_equal_ave(self, chain: int, nobs: int):
        self._c(self.lib.z2_obs_equal_ave(self.h, chain, nobs))

    def obs_tau_calc(self, chain: int, nt: int):
        self._c(self.lib.z2_obs_tau_calc(self.h, chain, nt))

    def obs_tau_ave(self, chain: int, nobst: int):
        self._c(self.lib.z2_obs_tau_ave(self.h, chain, nobst))

    def get_prop(self, chain: int) -> dict:
        """The Propagator: G, UR, DR, VR, UL, DL, VL (natural indexing)."""
        N = self.dims(chain)[0]
        m = {k: np.empty(N * N) for k in ("G", "UR", "VR", "UL", "VL")}
        d = {k: np.empty(N) for k in ("DR", "DL")}
        self._c(self.lib.z2_get_prop(self.h, chain, dptr(m["G"]), dptr(m["UR"]), dptr(d["DR"]),
                                     dptr(m["VR"]), dptr(m["UL"]), dptr(d["DL"]),
                                     dptr(m["VL"])))
        out = {k: v.reshape(N, N).T.copy() for k, v in m.items()}
        out.update(d)
        return out

    def set_prop(self, chain: int, G=None, UR=None, DR=None, VR=None, UL=None, DL=None,
                 VL=None):
        """Load any of the Propagator's matrices (None leaves one unchanged)."""
        given = {k: v for k, v in dict(G=G, UR=UR, DR=DR, VR=VR, UL=UL, DL=DL, VL=VL).items()
                 if v is not None}
        bufs = dict(zip(given, self._mats(chain, **given)))
        ptr = {k: (dptr(bufs[k]) if k in bufs else None)
               for k in ("G", "UR", "DR", "VR", "UL", "DL", "VL")}
        self._c(self.lib.z2_set_prop(self.h, chain, ptr["G"], ptr["UR"], ptr["DR"], ptr["VR"],
                                     ptr["UL"], ptr["DL"], ptr["VL"]))

    def get_propgr(self, chain: int) -> dict:
        """PropGreen of the time-displaced chain: G00, G0t, Gt0, Gtt."""
        N = self.dims(chain)[0]
        m = {k: np.empty(N * N) for k in ("G00", "G0t", "Gt0", "Gtt")}
        self._c(self.lib.z2_get_propgr(self.h, chain, *[dptr(v) for v in m.values()]))
        return {k: v.reshape(N, N).T.copy() for k, v in m.items()}
