"""CPU oracle for the Z2-gauge DQMC hot path (TEST INFRASTRUCTURE ONLY).

This module restates, in NumPy/SciPy, the reference Fortran routines of the
local DQMC sweep of SONY932/z2_gauge_zfy.  It exists to check the CUDA
library: only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg may import it.  The product path never routes through it.

Every function cites the reference routine it follows (paths are relative to
the reference project root).  Numerics:

* The reference stores every fermion matrix as ``complex(kind=8)`` but every
  entry is real (sigma, t, mu are real and ``NB_field = 0``,
  ``src/calc_basic.f90:47``).  The oracle therefore runs in real float64 by
  default (``dtype=np.float64``); ``dtype=np.complex128`` reruns the same
  algorithm with the complex LAPACK routines the reference calls
  (ZGEQP3/ZUNGQR/ZUNMQR/ZTRMM/ZTRSM) so that tests can show the imaginary
  parts stay exactly zero and the two agree to rounding.
* Spin up and spin down are built by the same operation sequence
  (``src/localK.f90:84-165``, ``src/multiply.f90``), so they are bit-identical;
  the oracle keeps one sector and squares the determinant ratio exactly as
  ``ratio_fermion = ProddetU * ProddetD`` does (``src/localK.f90:118``).
* LAPACK routines are SciPy's reference-LAPACK builds (dgeqp3 etc.), i.e. the
  same algorithms the reference links with ``-llapack``.  The NAG QR
  (F01RCF/F01REF) used by ``UDV_C`` and the LINPACK inverse (ZGEFA/ZGEDI)
  used by ``INV_C`` are not in SciPy; they are replaced by Householder QR
  (dgeqrf/dorgqr via numpy) and LU inversion (getrf/getri via numpy), which
  give the same Green's functions to rounding because the time-displaced
  Green's function does not depend on the QR convention.

Parity status: pinned against the reference's own recorded run.  The
reference cannot be compiled here (no Fortran compiler, no MPI), but its
test_run/ directory holds the output of its own binary for one 100-bin run
(global Wolff moves plus local sweeps, 4x4, Ltrot = 40, absolute = 5).
Replayed from the same inputs, this oracle reproduces that run's six per-bin
observable series to 2.3e-14 relative and its acceptance ratios, cluster size
and drift figures to the printed digits, which requires every accept/reject
decision to agree (tests/test_oracle_testrun.py, fixture extracted by
tests/golden/make_testrun_golden.py).  Known-answer tests built from the
algorithm itself (ranf closed form, free-fermion limit, dense-product
Green's function, mu-derivative identity, complex/real agreement, lattice
invariants) cover what that run does not reach; see tests/test_oracle.py.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.linalg import blas, lapack

RATIO_EPS = 1.0e-300   # src/globalK.f90:9
ZERO = 1.0e-10          # src/calc_basic.f90:5
UPBOUND = 1.0e200       # src/calc_basic.f90:7
IP_RANF = 48828125      # lib/package_of_matrix/Ran/ran_imada.f:60
TWO31 = 2 ** 31


# --------------------------------------------------------------------------
# Random numbers
# --------------------------------------------------------------------------
def ranf_step(iq: int) -> tuple[float, int]:
    """One call of ``ranf(iq)`` (lib/package_of_matrix/Ran/ran_imada.f:55-68).

    ``iq = iq*IP`` wraps in 32-bit signed arithmetic and a negative result is
    folded by ``iq = (iq+IR)+1``; together that is ``iq*IP mod 2**31``.
    Returns (value in [0,1), new state).
    """
    x = (iq * IP_RANF) & 0xFFFFFFFF
    if x >= TWO31:
        x -= 2 ** 32                     # signed 32-bit view
    if x < 0:
        x = (x + 2147483647) + 1          # ran_imada.f:65
    return x / 2.0 ** 31, x


class Ranf:
    """Stateful ``ranf`` stream; ``state`` is the Fortran ``iseed``."""

    def __init__(self, seed: int):
        self.state = int(seed)
        self.ndraws = 0

    def __call__(self) -> float:
        v, self.state = ranf_step(self.state)
        self.ndraws += 1
        return v


class ReplayStream:
    """A fixed sequence of uniforms used in place of ``ranf`` (replay tests)."""

    def __init__(self, values):
        self.values = np.asarray(values, dtype=np.float64)
        self.ndraws = 0

    def __call__(self) -> float:
        v = float(self.values[self.ndraws])
        self.ndraws += 1
        return v


# --------------------------------------------------------------------------
# Parameters (src/calc_basic.f90)
# --------------------------------------------------------------------------
@dataclass
class Params:
    """Input of ``read_input`` + ``Params_set`` (src/calc_basic.f90:50-102).

    ``RT`` may be a scalar (the reference) or a length-2N array of per-bond
    hopping amplitudes (used only by the log-det adjoint).
    """
    RT: object = 1.0
    J: float = 0.5
    h: float = 0.5
    mu: float = 0.0
    Q: float = 1.0
    Nlx: int = 4
    Nly: int = 4
    Ltrot: int = 40
    beta: float = 4.0
    NlxTherm: int | None = None
    NlyTherm: int | None = None
    LtrotTherm: int | None = None
    Nwrap: int = 10
    Nbin: int = 1
    Nsweep: int = 1
    is_tau: bool = False
    Nthermal: int = 0
    is_warm: bool = False
    Nwarm: int = 0
    is_global: bool = False
    Nglobal: int = 0
    absolute: int = 1

    def __post_init__(self):
        if self.NlxTherm is None:
            self.NlxTherm = self.Nlx
        if self.NlyTherm is None:
            self.NlyTherm = self.Nly
        if self.LtrotTherm is None:
            self.LtrotTherm = self.Ltrot
        # Params_set (src/calc_basic.f90:91-102)
        self.Lq = self.Nlx * self.Nly
        self.LqTherm = self.NlxTherm * self.NlyTherm
        self.dtau = self.beta / float(self.Ltrot)
        self.Ndim = self.Lq
        if self.Ltrot % self.Nwrap != 0:
            raise ValueError("Ltrot must be a multiple of Nwrap")
        self.Nst = self.Ltrot // self.Nwrap

    def rt_bond(self) -> np.ndarray:
        """Hopping amplitude per bond (uniform RT in the reference)."""
        if np.ndim(self.RT) == 0:
            return np.full(2 * self.Lq, float(self.RT))
        rt = np.asarray(self.RT, dtype=np.float64)
        assert rt.shape == (2 * self.Lq,)
        return rt

    def rt_scalar(self) -> float:
        """RT as used by observables and the ``RT > Zero`` tests."""
        if np.ndim(self.RT) == 0:
            return float(self.RT)
        return float(np.mean(self.RT))


def read_params(path: str) -> Params:
    """Parse ``paramC_sets.txt`` in the order of ``read_input``
    (src/calc_basic.f90:52-62)."""
    def logical(tok: str) -> bool:
        t = tok.strip().lower().strip(".")
        return t in ("true", "t")

    with open(path) as f:
        lines = [ln for ln in f.read().splitlines() if ln.strip()][:8]
    t = [ln.split() for ln in lines]
    return Params(
        RT=float(t[0][0]), J=float(t[0][1]), h=float(t[0][2]), mu=float(t[0][3]),
        Q=float(t[0][4]),
        Nlx=int(t[1][0]), Nly=int(t[1][1]), Ltrot=int(t[1][2]), beta=float(t[1][3]),
        NlxTherm=int(t[2][0]), NlyTherm=int(t[2][1]), LtrotTherm=int(t[2][2]),
        Nwrap=int(t[3][0]), Nbin=int(t[3][1]), Nsweep=int(t[3][2]),
        is_tau=logical(t[4][0]), Nthermal=int(t[4][1]),
        is_warm=logical(t[5][0]), Nwarm=int(t[5][1]),
        is_global=logical(t[6][0]), Nglobal=int(t[6][1]),
        absolute=int(t[7][0]))


def npbc(nr: int, L: int) -> int:
    """Periodic wrap of a 1-based coordinate (src/calc_basic.f90:124-130)."""
    if nr < 1:
        return nr + L
    if nr > L:
        return nr - L
    return nr


# --------------------------------------------------------------------------
# Lattice (src/lattice.f90:25-221), 0-based indices, same enumeration
# --------------------------------------------------------------------------
class Lattice:
    def __init__(self, Nlx: int, Nly: int):
        self.Nlx, self.Nly = Nlx, Nly
        Lq = Nlx * Nly
        self.Lq = Lq
        # n_list / inv_n_list (lattice.f90:31-40): site = (y-1)*Lx + (x-1)
        self.n_list = np.zeros((Lq, 2), dtype=np.int64)          # 1-based x, y
        self.inv_n_list = np.zeros((Nlx + 1, Nly + 1), dtype=np.int64)
        nc = 0
        for ny in range(1, Nly + 1):
            for nx in range(1, Nlx + 1):
                self.n_list[nc] = (nx, ny)
                self.inv_n_list[nx, ny] = nc
                nc += 1
        inv = self.inv_n_list
        # bond_list (lattice.f90:42-60): bond 2*i = +x of site i, 2*i+1 = +y
        self.bond_list = np.zeros((2 * Lq, 2), dtype=np.int64)
        self.inv_bond_list = -np.ones((Lq, Lq), dtype=np.int64)
        nc = 0
        for ny in range(1, Nly + 1):
            for nx in range(1, Nlx + 1):
                ii = inv[nx, ny]
                ix = inv[npbc(nx + 1, Nlx), ny]
                self.bond_list[nc] = (ii, ix)
                self.inv_bond_list[ii, ix] = nc
                nc += 1
                iy = inv[nx, npbc(ny + 1, Nly)]
                self.bond_list[nc] = (ii, iy)
                self.inv_bond_list[ii, iy] = nc
                nc += 1
        # checkerboard groups (lattice.f90:72-102)
        g = [[], [], [], []]
        for nc in range(2 * Lq):
            ii, jj = self.bond_list[nc]
            ixc, iyc = self.n_list[ii]
            jxc, jyc = self.n_list[jj]
            if npbc(ixc + 1, Nlx) == jxc:
                g[0 if ixc % 2 == 0 else 1].append(nc)
            elif npbc(iyc + 1, Nly) == jyc:
                g[2 if iyc % 2 == 0 else 3].append(nc)
        self.groups = [np.array(x, dtype=np.int64) for x in g]
        self.group_disjoint = []
        for grp in self.groups:
            sites = self.bond_list[grp].ravel()
            self.group_disjoint.append(len(set(sites.tolist())) == len(sites))
        # plaquette partner bonds (lattice.f90:104-141)
        bb = np.zeros((2 * Lq, 7), dtype=np.int64)
        ib = self.inv_bond_list
        for nc in range(2 * Lq):
            ii, jj = self.bond_list[nc]
            ixc, iyc = self.n_list[ii]
            jxc, jyc = self.n_list[jj]
            bb[nc, 0] = nc
            if npbc(ixc + 1, Nlx) == jxc:
                nx = inv[ixc, npbc(iyc + 1, Nly)]
                bb[nc, 1] = ib[ii, nx]
                ny = inv[jxc, npbc(jyc + 1, Nly)]
                bb[nc, 2] = ib[nx, ny]
                bb[nc, 3] = ib[jj, ny]
                nx = inv[ixc, npbc(iyc - 1, Nly)]
                bb[nc, 4] = ib[nx, ii]
                ny = inv[jxc, npbc(jyc - 1, Nly)]
                bb[nc, 5] = ib[nx, ny]
                bb[nc, 6] = ib[ny, jj]
            elif npbc(iyc + 1, Nly) == jyc:
                nx = inv[npbc(jxc - 1, Nlx), jyc]
                bb[nc, 1] = ib[nx, jj]
                ny = inv[npbc(ixc - 1, Nlx), iyc]
                bb[nc, 2] = ib[ny, nx]
                bb[nc, 3] = ib[ny, ii]
                nx = inv[npbc(jxc + 1, Nlx), jyc]
                bb[nc, 4] = ib[jj, nx]
                ny = inv[npbc(ixc + 1, Nlx), iyc]
                bb[nc, 5] = ib[ny, nx]
                bb[nc, 6] = ib[ii, ny]
        self.bond_bonds = bb
        # imj (lattice.f90:144-155)
        self.imj = np.zeros((Lq, Lq), dtype=np.int64)
        for jj in range(Lq):
            for ii in range(Lq):
                ixc, iyc = self.n_list[ii]
                jxc, jyc = self.n_list[jj]
                self.imj[ii, jj] = inv[npbc(ixc - jxc, Nlx), npbc(iyc - jyc, Nly)]
        # momenta and phases (lattice.f90:158-176)
        self.xk_v = np.zeros((Lq, 2))
        self.aimj_v = np.zeros((Lq, 2))
        for ii in range(Lq):
            ixc, iyc = self.n_list[ii]
            self.aimj_v[ii] = (float(ixc), float(iyc))
            self.xk_v[ii] = (float(ixc - 1) * 2.0 * math.pi / Nlx,
                             float(iyc - 1) * 2.0 * math.pi / Nly)
        self.k_dot_r = self.xk_v @ self.aimj_v.T
        # nearest neighbours (lattice.f90:186-195)
        self.L_bonds = np.zeros((Lq, 5), dtype=np.int64)
        for iyc in range(1, Nly + 1):
            for ixc in range(1, Nlx + 1):
                ii = inv[ixc, iyc]
                self.L_bonds[ii] = (ii, inv[npbc(ixc + 1, Nlx), iyc],
                                    inv[ixc, npbc(iyc + 1, Nly)],
                                    inv[npbc(ixc - 1, Nlx), iyc],
                                    inv[ixc, npbc(iyc - 1, Nly)])

    def fourier_r_to_k(self, gr: np.ndarray) -> np.ndarray:
        """``FFT_RtoK_*`` (src/lattice.f90:247-333): naive DFT over the first
        axis, normalised by 1/Lq."""
        ph = np.exp(1j * self.k_dot_r)            # (nk, imj)
        return np.tensordot(ph, gr, axes=(1, 0)) / float(self.Lq)


# --------------------------------------------------------------------------
# Gauge configuration (src/fields.f90)
# --------------------------------------------------------------------------
def lambda_enforce_sector(lam: np.ndarray, Q: float) -> None:
    """src/fields.f90:580-603."""
    prod = 1.0
    for i in range(lam.size):
        lam[i] = 1.0 if lam[i] >= 0.0 else -1.0
        prod *= lam[i]
    target = 1.0 if Q >= 0.0 else -1.0
    if prod * target < 0.0:
        lam[-1] = -lam[-1]


def lambda_random_fill(lam: np.ndarray, rng: Ranf, Q: float) -> None:
    """src/fields.f90:559-578."""
    for i in range(lam.size):
        lam[i] = 1.0 if rng() >= 0.5 else -1.0
    lambda_enforce_sector(lam, Q)


def conf_set(p: Params, rng: Ranf):
    """Initial sigma(2*LqTherm, LtrotTherm) and lambda(LqTherm)
    (src/fields.f90:311-427).  ``rng`` continues afterwards (the Fortran
    ``itmp`` is ``intent(inout)``)."""
    nb, lt = 2 * p.LqTherm, p.LtrotTherm
    sigma = np.zeros((nb, lt))
    if p.absolute == 1:
        for nt in range(lt):
            for ii in range(nb):
                sigma[ii, nt] = 1.0 if rng() >= 0.5 else -1.0
    elif p.absolute == 2:
        for nt in range(lt):
            for ii in range(nb):
                x1 = rng()
                x2 = rng()
                x = math.sqrt(-2.0 * math.log(x1)) * math.cos(2.0 * math.pi * x2)
                sigma[ii, nt] = 1.0 if x >= 0.0 else -1.0
    elif p.absolute == 3:
        sigma[:] = 1.0
    elif p.absolute == 4:
        Lx = p.NlxTherm
        for nc in range(nb):
            site = nc // 2
            nx, ny = site % Lx + 1, site // Lx + 1
            sigma[nc, :] = 1.0 if (nx + ny) % 2 == 0 else -1.0
    elif p.absolute == 5:
        for ii in range(nb):
            sigma[ii, :] = 1.0 if rng() >= 0.5 else -1.0
    else:
        raise ValueError(f"incorrect absolute input {p.absolute}")
    lam = np.zeros(p.LqTherm)
    lambda_random_fill(lam, rng, p.Q)
    return sigma, lam


def conf_transfer(p: Params, lat: Lattice, sigma_therm, lambda_therm):
    """Tile a thermalisation-size configuration up to the run size
    (src/fields.f90:429-507)."""
    sigma = np.zeros((2 * p.Lq, p.Ltrot))
    for nt in range(p.LtrotTherm):
        for b in range(2 * p.Lq):
            ii, jj = lat.bond_list[b]
            nx, ny = lat.n_list[ii]
            jx, jy = lat.n_list[jj]
            nxt = (nx - 1) % p.NlxTherm + 1
            nyt = (ny - 1) % p.NlyTherm + 1
            if npbc(nx + 1, p.Nlx) == jx:
                bt = (nyt - 1) * p.NlxTherm * 2 + (nxt - 1) * 2 + 1
            else:
                bt = (nyt - 1) * p.NlxTherm * 2 + (nxt - 1) * 2 + 2
            sigma[b, nt] = sigma_therm[bt - 1, nt]
    for nt in range(p.LtrotTherm, p.Ltrot):
        sigma[:, nt] = sigma[:, nt - p.LtrotTherm]
    lam = np.zeros(p.Lq)
    for ii in range(p.Lq):
        nx, ny = lat.n_list[ii]
        nxt = (nx - 1) % p.NlxTherm + 1
        nyt = (ny - 1) % p.NlyTherm + 1
        lam[ii] = lambda_therm[(nyt - 1) * p.NlxTherm + nxt - 1]
    lambda_enforce_sector(lam, p.Q)
    return sigma, lam


def seeded_config(p: Params, lat: Lattice, seed: int):
    """Fresh start from ``seeds.txt`` on one rank: ``conf_set`` then
    ``conf_transfer`` (src/fields.f90:250-264, 214-225).  Returns sigma,
    lambda and the RNG whose state continues as ``iseed``."""
    rng = Ranf(seed)
    st, lt = conf_set(p, rng)
    sigma, lam = conf_transfer(p, lat, st, lt)
    return sigma, lam, rng


def boson_ratio_local(p: Params, lat: Lattice, sigma: np.ndarray, ii: int,
                      nt: int, s_new: float) -> float:
    """``m_bosonratio_local`` (src/fields.f90:40-119); ``nt`` is 0-based."""
    alpha = p.dtau * p.J
    if abs(p.h) > ZERO:
        tanh_arg = math.tanh(p.dtau * p.h)
        if tanh_arg < 1.0e-300:
            tanh_arg = 1.0e-300
        gamma = -0.5 * math.log(tanh_arg)
        use_temporal = True
    else:
        gamma = 0.0
        use_temporal = False
    log_upbound = math.log(UPBOUND)
    bb = lat.bond_bonds[ii]
    tmp = s_new
    for nf in (1, 2, 3):
        tmp = tmp * sigma[bb[nf], nt]
    tmp_new = 0.0 + tmp
    tmp = s_new
    for nf in (4, 5, 6):
        tmp = tmp * sigma[bb[nf], nt]
    tmp_new = tmp_new + tmp
    s_old = sigma[ii, nt]
    tmp = s_old
    for nf in (1, 2, 3):
        tmp = tmp * sigma[bb[nf], nt]
    tmp_old = 0.0 + tmp
    tmp = s_old
    for nf in (4, 5, 6):
        tmp = tmp * sigma[bb[nf], nt]
    tmp_old = tmp_old + tmp
    expo = alpha * (tmp_new - tmp_old)
    expo = min(max(expo, -log_upbound), log_upbound)
    ratio = math.exp(expo)
    if use_temporal:
        tmp_new = 0.0
        tmp_old = 0.0
        L = p.Ltrot
        for nf in (-1, 1):
            ntn = (nt + nf) % L
            tmp_new = tmp_new + s_new * sigma[ii, ntn]
            tmp_old = tmp_old + s_old * sigma[ii, ntn]
        expo = gamma * (tmp_new - tmp_old)
        expo = min(max(expo, -log_upbound), log_upbound)
        ratio = ratio * math.exp(expo)
    return ratio


# --------------------------------------------------------------------------
# Checkerboard kinetic operator (src/operator_kin.f90)
# --------------------------------------------------------------------------
GROUP_ORDER = (0, 1, 2, 3, 3, 2, 1, 0)   # operator_kin.f90:75-85, 107-117


class OperatorKin:
    """``OperatorKin`` (src/operator_kin.f90:7-19) with per-bond alpha."""

    def __init__(self, p: Params, lat: Lattice):
        self.p, self.lat = p, lat
        rt = p.rt_bond()
        self.alpha = 0.5 * p.dtau * rt          # opK_set, operator_kin.f90:26
        self.alpha_2 = p.dtau * rt              # operator_kin.f90:27

    def get_delta(self, b: int, s_old: float, s_new: float) -> np.ndarray:
        """``opK_get_delta`` (src/operator_kin.f90:40-59)."""
        a2 = self.alpha_2[b]
        c_new = math.cosh(a2 * s_new)
        c_old = math.cosh(a2 * s_old)
        s_n = math.sinh(a2 * s_new)
        s_o = math.sinh(a2 * s_old)
        d = np.empty((2, 2))
        d[0, 0] = c_new * c_old - s_n * s_o - 1.0
        d[0, 1] = s_n * c_old - c_new * s_o
        d[1, 0] = s_n * c_old - c_new * s_o
        d[1, 1] = c_new * c_old - s_n * s_o - 1.0
        return d

    def _cs(self, grp, sigma, nt, nflag):
        x = nflag * self.alpha[grp] * sigma[grp, nt]
        return np.cosh(x), np.sinh(x)

    def process_group(self, M, g, sigma, nt, nflag):
        """Row rotations of one group (src/operator_kin.f90:88-120)."""
        grp = self.lat.groups[g]
        C, S = self._cs(grp, sigma, nt, nflag)
        p1 = self.lat.bond_list[grp, 0]
        p2 = self.lat.bond_list[grp, 1]
        if self.lat.group_disjoint[g]:
            a = M[p1, :].copy()
            b = M[p2, :].copy()
            M[p1, :] = C[:, None] * a + S[:, None] * b
            M[p2, :] = S[:, None] * a + C[:, None] * b
        else:
            for k in range(grp.size):
                a = M[p1[k], :].copy()
                b = M[p2[k], :].copy()
                M[p1[k], :] = C[k] * a + S[k] * b
                M[p2[k], :] = S[k] * a + C[k] * b

    def process_group_L(self, M, g, sigma, nt, nflag):
        """Column rotations of one group (src/operator_kin.f90:147-179)."""
        grp = self.lat.groups[g]
        C, S = self._cs(grp, sigma, nt, nflag)
        p1 = self.lat.bond_list[grp, 0]
        p2 = self.lat.bond_list[grp, 1]
        if self.lat.group_disjoint[g]:
            a = M[:, p1].copy()
            b = M[:, p2].copy()
            M[:, p1] = a * C[None, :] + b * S[None, :]
            M[:, p2] = a * S[None, :] + b * C[None, :]
        else:
            for k in range(grp.size):
                a = M[:, p1[k]].copy()
                b = M[:, p2[k]].copy()
                M[:, p1[k]] = a * C[k] + b * S[k]
                M[:, p2[k]] = a * S[k] + b * C[k]

    def mmult_R(self, M, sigma, nt, nflag):
        """M <- B_nt^{nflag} M (src/operator_kin.f90:61-86); nt 0-based."""
        for g in GROUP_ORDER:
            self.process_group(M, g, sigma, nt, nflag)

    def mmult_L(self, M, sigma, nt, nflag):
        """M <- M B_nt^{nflag} (src/operator_kin.f90:122-145); nt 0-based."""
        for g in GROUP_ORDER:
            self.process_group_L(M, g, sigma, nt, nflag)

    def dense_B(self, sigma, nt, nflag=1, dtype=np.float64):
        M = np.eye(self.p.Lq, dtype=dtype)
        self.mmult_R(M, sigma, nt, nflag)
        return M


class OperatorMU:
    """``OperatorMU`` (src/non_interact.f90:19-57): a scalar factor."""

    def __init__(self, p: Params):
        self.expMU_P = math.exp(p.dtau * p.mu)
        self.expMU_M = math.exp(-p.dtau * p.mu)

    def factor(self, nflag):
        return self.expMU_P if nflag == 1 else self.expMU_M


# --------------------------------------------------------------------------
# Propagator state (src/process_matrix.f90)
# --------------------------------------------------------------------------
class Propagator:
    """``Propagator`` (src/process_matrix.f90:6-15, 46-56)."""

    def __init__(self, N, dtype=np.float64):
        I = np.eye(N, dtype=dtype)
        self.UUR, self.VUR, self.DUR = I.copy(), I.copy(), np.ones(N)
        self.UUL, self.VUL, self.DUL = I.copy(), I.copy(), np.ones(N)
        self.Gr = I.copy()
        self.Xmaxm = 0.0
        self.Xmeanm = 0.0

    def copy(self):
        c = Propagator.__new__(Propagator)
        for k, v in self.__dict__.items():
            c.__dict__[k] = v.copy() if isinstance(v, np.ndarray) else v
        return c


class WrapList:
    """``WrapList`` (src/process_matrix.f90:26-33, 104-112)."""

    def __init__(self, N, Nst, dtype=np.float64):
        z = lambda: np.zeros((Nst + 1, N, N), dtype=dtype)
        self.URlist, self.VRlist, self.ULlist, self.VLlist = z(), z(), z(), z()
        self.DRlist = np.zeros((Nst + 1, N))
        self.DLlist = np.zeros((Nst + 1, N))


def _wrlist_copy(wr: "WrapList") -> "WrapList":
    c = WrapList.__new__(WrapList)
    for k, v in wr.__dict__.items():
        c.__dict__[k] = v.copy()
    return c


class PropGreen:
    """``PropGreen`` (src/process_matrix.f90:17-24, 68-96)."""

    def __init__(self, G):
        self.reset(G)
        self.Xmaxm = np.zeros(3)
        self.Xmeanm = np.zeros(3)

    def reset(self, G):
        I = np.eye(G.shape[0], dtype=G.dtype)
        self.Gr00 = G.copy()
        self.Grtt = G.copy()
        self.Grt0 = G.copy()
        self.Gr0t = -(I - G)


# --------------------------------------------------------------------------
# Stabilization (src/stabilization.f90)
# --------------------------------------------------------------------------
def _ct(A):
    return np.conj(A.T) if np.iscomplexobj(A) else A.T.copy()


def _lapack(dtype, name):
    pre = "z" if np.dtype(dtype) == np.complex128 else "d"
    mod = blas if name in ("trmm", "trsm") else lapack
    if name == "orgqr" and pre == "z":
        name = "ungqr"
    if name == "ormqr" and pre == "z":
        name = "unmqr"
    return getattr(mod, pre + name)


def qdrp_decompose(M):
    """``QDRP_decompose`` (src/stabilization.f90:42-68): pivoted QR,
    D = |R_ii|, rows of R divided by D.  Returns (qr, D, jpvt(1-based), tau)."""
    N = M.shape[0]
    geqp3 = _lapack(M.dtype, "geqp3")
    qr, jpvt, tau, work, info = geqp3(M, lwork=max(64 * N, 1))
    assert info == 0
    qr = np.array(qr, order="F")
    D = np.empty(N)
    for i in range(N):
        x = abs(qr[i, i])
        D[i] = x
        qr[i, i:] = qr[i, i:] / x
    return qr, D, np.asarray(jpvt, dtype=np.int64), tau


def lapmr_forward(X, jpvt):
    """ZLAPMR(.true.): row I of the result is row jpvt(I) of X."""
    return X[jpvt - 1, :].copy()


def lapmr_backward(X, jpvt):
    """ZLAPMR(.false.): row I of X moves to row jpvt(I)."""
    Y = np.empty_like(X)
    Y[jpvt - 1, :] = X
    return Y


def lapmt_forward(X, jpvt):
    """ZLAPMT(.true.): column J of the result is column jpvt(J) of X."""
    return X[:, jpvt - 1].copy()


def lapmt_backward(X, jpvt):
    """ZLAPMT(.false.): column J of X moves to column jpvt(J)."""
    Y = np.empty_like(X)
    Y[:, jpvt - 1] = X
    return Y


def stab_UR(prop: Propagator):
    """src/stabilization.f90:70-94."""
    dt = prop.UUR.dtype
    mat = prop.UUR * prop.DUR[None, :]
    qr, D, jpvt, tau = qdrp_decompose(mat)
    prop.DUR = D
    V = lapmr_forward(prop.VUR, jpvt)
    trmm = _lapack(dt, "trmm")
    prop.VUR = trmm(1.0, qr, V, side=0, lower=0, trans_a=0, diag=0)
    orgqr = _lapack(dt, "orgqr")
    q, work, info = orgqr(qr, tau, lwork=max(64 * qr.shape[0], 1))
    assert info == 0
    prop.UUR = np.array(q)


def stab_UL(prop: Propagator):
    """src/stabilization.f90:96-120."""
    dt = prop.UUL.dtype
    mat = _ct(prop.UUL) * prop.DUL[None, :]
    qr, D, jpvt, tau = qdrp_decompose(mat)
    prop.DUL = D
    V = lapmt_forward(prop.VUL, jpvt)
    trmm = _lapack(dt, "trmm")
    prop.VUL = trmm(1.0, qr, V, side=1, lower=0, trans_a=2 if dt == np.complex128 else 1, diag=0)
    orgqr = _lapack(dt, "orgqr")
    q, work, info = orgqr(qr, tau, lwork=max(64 * qr.shape[0], 1))
    assert info == 0
    prop.UUL = _ct(np.array(q))


def stab_green(prop: Propagator, nt: int, Ltrot: int):
    """G = (I + UR DR VR VL DL UL)^{-1} (src/stabilization.f90:122-200).
    ``nt`` is the Fortran time-slice number (0..Ltrot)."""
    dt = prop.UUR.dtype
    N = prop.UUR.shape[0]
    VRVL = prop.VUR @ prop.VUL
    invULUR = _ct(prop.UUR) @ _ct(prop.UUL)
    temp = VRVL * prop.DUL[None, :]
    VRVL = prop.DUR[:, None] * temp
    mat = invULUR + VRVL
    half = Ltrot // 2
    if nt > half:
        mat = _ct(mat)
    qr, D, jpvt, tau = qdrp_decompose(mat)
    ormqr = _lapack(dt, "ormqr")
    trsm = _lapack(dt, "trsm")
    cflag = b"C" if dt == np.complex128 else b"T"
    lw = max(64 * N, 1)
    if nt < half + 1:
        temp = _ct(prop.UUR)
        temp, work, info = ormqr(b"L", cflag, qr, tau, temp, lw)
        assert info == 0
        temp = temp / D[:, None]
        temp = trsm(1.0, qr, temp, side=0, lower=0, trans_a=0, diag=0)
        temp = lapmr_backward(temp, jpvt)
        G = _ct(prop.UUL) @ temp
    else:
        temp = _ct(prop.UUL)
        temp, work, info = ormqr(b"R", b"N", qr, tau, temp, lw)
        assert info == 0
        temp = temp / D[None, :]
        temp = trsm(1.0, qr, temp, side=1, lower=0,
                    trans_a=2 if dt == np.complex128 else 1, diag=0)
        temp = lapmt_backward(temp, jpvt)
        G = temp @ _ct(prop.UUR)
    return np.array(G)


def udv_nag(A):
    """``UDV_C`` (lib/package_of_matrix/Modules/mat_mod.f90:604-711) with the
    NAG QR replaced by Householder QR: A = U diag(D) V, V unit-diagonal-
    normalised upper triangular, with the determinant-sign fix of
    mat_mod.f90:650-657."""
    Q, R = np.linalg.qr(A)
    detv = np.prod(np.real(np.diag(R)))
    if detv < 0.0:
        Q[:, 0] = -Q[:, 0]
        R[0, :] = -R[0, :]
    D = np.abs(np.real(np.diag(R)))
    V = R / D[:, None]
    return Q, D, V


def stab_green_big(prop: Propagator):
    """Time-displaced Green's functions from the 2N x 2N block matrix
    (src/stabilization.f90:202-264).  Returns Gr00, Gr0t, Grt0, Grtt."""
    N = prop.UUR.shape[0]
    inv = np.linalg.inv
    ULUR = prop.UUL @ prop.UUR
    VRVL = prop.VUR @ prop.VUL
    invULUR = inv(ULUR)
    invVRVL = inv(VRVL)
    big = np.zeros((2 * N, 2 * N), dtype=prop.UUR.dtype)
    big[:N, :N] = invVRVL
    big[N:, N:] = invULUR
    idx = np.arange(N)
    big[idx, idx + N] = prop.DUL
    big[idx + N, idx] = -prop.DUR
    bigU, bigD, bigV = udv_nag(big)
    invbigU, invbigV = inv(bigU), inv(bigV)
    invUUR, invUUL = inv(prop.UUR), inv(prop.UUL)
    invVUR, invVUL = inv(prop.VUR), inv(prop.VUL)
    left = np.zeros_like(big)
    left[:N, :N] = invVUR
    left[N:, N:] = invUUL
    mat_left = left @ invbigV
    right = np.zeros_like(big)
    right[:N, :N] = invVUL
    right[N:, N:] = invUUR
    mat_right = invbigU @ right
    mat_left = mat_left / bigD[None, :]
    tot = mat_left @ mat_right
    return (tot[:N, :N].copy(), tot[:N, N:].copy(), tot[N:, :N].copy(),
            tot[N:, N:].copy())


def compare_mat(A, B) -> float:
    """src/stabilization.f90:365-372."""
    return float(np.max(np.abs(A - B)))


# --------------------------------------------------------------------------
# Observables (src/obser_equal.f90, src/obser_tau.f90)
# --------------------------------------------------------------------------
class ObserEqual:
    """src/obser_equal.f90:7-149."""

    def __init__(self, p: Params, lat: Lattice):
        self.p, self.lat = p, lat
        self.reset()
        Lq = p.Lq
        n = lat.n_list
        self.stag = np.where((n[:, 0] + n[:, 1]) % 2 == 0, 1.0, -1.0)
        qx = math.pi - 2.0 * math.pi / float(p.Nlx)
        dx = (n[:, 0][:, None] - n[:, 0][None, :]).astype(np.float64)
        dy = (n[:, 1][:, None] - n[:, 1][None, :]).astype(np.float64)
        self.phase_shift = np.cos(qx * dx + math.pi * dy)
        self.phase_pi = self.stag[:, None] * self.stag[None, :]
        # plaquette bonds (obser_equal.f90:46-55)
        pl = []
        for site in range(Lq):
            right = lat.L_bonds[site, 1]
            up = lat.L_bonds[site, 2]
            diag = lat.L_bonds[up, 1]
            ib = lat.inv_bond_list
            pl.append((ib[site, right], ib[right, lat.L_bonds[right, 2]],
                       ib[up, diag], ib[site, up]))
        self.plaq = np.array(pl, dtype=np.int64)

    def reset(self):
        """src/obser_equal.f90:33-48."""
        self.flux_sum = self.flux_sq = 0.0
        self.flux_avg = self.chi_flux = 0.0
        self.pair_sc_acc = self.pair_sc_q0 = 0.0
        self.cdw_pi_acc = self.cdw_shift_acc = 0.0
        self.cdw_pi = self.cdw_shift = self.cdw_ratio = 0.0
        self.density = 0.0

    def slice_values(self, G, sigma, nt):
        """Per-slice sums of ``Obs_equal_calc`` (src/obser_equal.f90:73-149):
        flux_tau, pair_sum, cdw_sum, cdw_shift_sum, density_slice."""
        Lq = self.p.Lq
        s = sigma[:, nt]
        pl = self.plaq
        flux = float(np.sum(s[pl[:, 0]] * s[pl[:, 1]] * s[pl[:, 2]] * s[pl[:, 3]])) / float(Lq)
        Gu = np.real(G)
        n_i = 1.0 - np.diag(Gu)
        dens = float(np.sum(n_i + n_i))
        I = np.eye(Lq)
        pair = float(np.sum((I - Gu) * (I - Gu)))
        # density_corr(i,j) for identical spin sectors
        nn = n_i[:, None] * n_i[None, :]
        exch = (I - Gu.T) * Gu
        corr = (nn - exch) + (nn - exch) + nn + nn
        cdw = float(np.sum(self.phase_pi * corr))
        cdws = float(np.sum(self.phase_shift * corr))
        return flux, pair, cdw, cdws, dens / float(Lq)

    def calc(self, G, sigma, nt):
        flux, pair, cdw, cdws, dens = self.slice_values(G, sigma, nt)
        self.flux_sum += flux
        self.flux_sq += flux * flux
        self.pair_sc_acc += pair
        self.cdw_pi_acc += cdw
        self.cdw_shift_acc += cdws
        self.density += dens

    def ave(self, Nobs):
        """src/obser_equal.f90:50-71."""
        if Nobs <= 0:
            return
        Lq = self.p.Lq
        z = 1.0 / float(Nobs)
        fm = self.flux_sum * z
        fsq = self.flux_sq * z
        self.flux_avg = fm
        self.chi_flux = self.p.beta * float(Lq) * max(0.0, fsq - fm * fm)
        self.pair_sc_q0 = (self.pair_sc_acc * z) / float(Lq)
        self.cdw_pi = (self.cdw_pi_acc * z) / float(Lq)
        self.cdw_shift = (self.cdw_shift_acc * z) / float(Lq)
        self.cdw_ratio = 1.0 - self.cdw_shift / self.cdw_pi if self.cdw_pi > 1.0e-12 else 0.0
        self.density = self.density * z

    def as_dict(self):
        return dict(flux_avg=self.flux_avg, chi_flux=self.chi_flux,
                    pair_sc_q0=self.pair_sc_q0, cdw_pi=self.cdw_pi,
                    cdw_shift=self.cdw_shift, cdw_ratio=self.cdw_ratio,
                    density=self.density)


TAU_NAMES = ("spin", "single", "pair_d", "pair_s", "charge_d", "charge_s", "curxx")


class ObserTau:
    """src/obser_tau.f90:7-133 (arrays indexed [imj, nt])."""

    def __init__(self, p: Params, lat: Lattice):
        self.p, self.lat = p, lat
        self.reset()

    def reset(self):
        z = lambda: np.zeros((self.p.Lq, self.p.Ltrot), dtype=np.complex128)
        self.arr = {k: z() for k in TAU_NAMES}

    def ave(self, Nobst):
        for k in TAU_NAMES:
            self.arr[k] = self.arr[k] * (1.0 / float(Nobst))

    def calc(self, pg: PropGreen, sigma, nt):
        """Literal per-tau accumulation with both (identical) spin sectors;
        ``nt`` is 0-based (Fortran ntau = nt+1)."""
        lat = self.lat
        Lq = self.p.Lq
        RT = self.p.rt_scalar()
        I = np.eye(Lq)
        g00 = pg.Gr00.astype(np.complex128)
        gtt = pg.Grtt.astype(np.complex128)
        gt0 = pg.Grt0.astype(np.complex128)
        g0t = pg.Gr0t.astype(np.complex128)
        g00c = I - g00.T
        gttc = I - gtt.T
        tmp_t = np.diag(gttc) + np.conj(np.diag(gttc))
        tmp_0 = np.diag(g00c) + np.conj(np.diag(g00c))
        imj = lat.imj
        a = self.arr
        # tmp_t_u == tmp_t_d and tmp_0_u == tmp_0_d for identical sectors
        spin = np.outer(sigma[:Lq, nt], sigma[:Lq, 0]).astype(np.complex128)
        d = g0t.T * np.conj(g0t.T)             # diag(ii,jj) = Gr0t(jj,ii)*conj
        pair = (d + d) * 4.0
        x = g0t.T * gt0                        # Gr0t(jj,ii)*Grt0(ii,jj)
        ch_common = -x - np.conj(x) - x - np.conj(x)
        ch_d = ch_common + np.outer(tmp_t - tmp_t, tmp_0 - tmp_0)
        ch_s = ch_common + np.outer(tmp_t + tmp_t, tmp_0 + tmp_0)
        term = gt0 + gt0
        single = term + np.conj(term)
        ip = lat.L_bonds[:, 1]
        # curxx (obser_tau.f90:107-131) with NB_field = 0 (all phases 1)
        cur = np.zeros((Lq, Lq), dtype=np.complex128)
        for jj in range(Lq):
            jp = ip[jj]
            for ii in range(Lq):
                ipp = ip[ii]
                term_c = (-g0t[jj, ipp] * gt0[ii, jp] - g0t[jp, ii] * gt0[ipp, jj]
                          + g0t[jj, ii] * gt0[ipp, jp] + g0t[jp, ipp] * gt0[ii, jj])
                x1 = -RT * RT * term_c - RT * RT * np.conj(term_c)
                cur[ii, jj] = x1 + x1           # spin up + spin down
        for name, val in (("spin", spin), ("pair_d", pair), ("pair_s", pair),
                          ("charge_d", ch_d), ("charge_s", ch_s),
                          ("single", single), ("curxx", cur)):
            np.add.at(a[name][:, nt], imj.ravel(), val.ravel())


def k_dot_r(lat: Lattice) -> np.ndarray:
    """Latt%k_dot_r (src/lattice.f90:159-173): xk_v(nk) = ((ix-1) 2pi/Nlx,
    (iy-1) 2pi/Nly), aimj_v(imj) = (ix, iy) (1-based), k_dot_r(nk, imj)."""
    xy = lat.n_list.astype(np.float64)
    kx = (xy[:, 0] - 1.0) * 2.0 * np.pi / lat.Nlx
    ky = (xy[:, 1] - 1.0) * 2.0 * np.pi / lat.Nly
    return np.outer(kx, xy[:, 0]) + np.outer(ky, xy[:, 1])


def fourier_r_to_k(gr: np.ndarray, lat: Lattice) -> np.ndarray:
    """FFT_RtoK_2 (src/lattice.f90:263-281): gk(nk, nf) = sum_imj
    exp(i k_dot_r(nk, imj)) gr(imj, nf) / Lq, summed in the reference's order
    (imj outer, one term at a time)."""
    kr = k_dot_r(lat)
    ph = np.exp(1j * kr)
    gk = np.zeros((lat.Lq, gr.shape[1]), dtype=np.complex128)
    for imj in range(lat.Lq):
        gk += ph[:, imj:imj + 1] * gr[imj:imj + 1, :]
    return gk / float(lat.Lq)


def integrate_susc(gk: np.ndarray, dtau: float) -> np.ndarray:
    """m_integrate_susc_2_mom (src/fourier_trans.f90:165-177)."""
    out = np.zeros(gk.shape[0], dtype=np.complex128)
    for nt in range(gk.shape[1]):
        out += gk[:, nt]
    return out * dtau


def integrate_susc_freq(gk: np.ndarray, dtau: float) -> np.ndarray:
    """m_integrate_susc_2_freq (src/fourier_trans.f90:179-191): Matsubara
    transform of the first momentum row."""
    L = gk.shape[1]
    out = np.zeros(L, dtype=np.complex128)
    for nw in range(L):
        for nt in range(L):
            out[nw] += np.exp(1j * 2.0 * np.pi * nt * nw / L) * gk[0, nt]
    return out * dtau


# --------------------------------------------------------------------------
# The model and the sweeps (src/localK.f90, src/local_sweep.f90,
# src/dynamics.f90, src/multiply.f90)
# --------------------------------------------------------------------------
class Z2Chain:
    """One Markov chain: the reference's module-global state of one MPI rank
    (src/model.f90:10-13, src/local_sweep.f90:27-29) plus PropU/WrU of
    src/main.f90:20-21 (one spin sector)."""

    def __init__(self, p: Params, sigma=None, seed: int = 12345, rng=None,
                 dtype=np.float64, record_decisions=False):
        self.p = p
        self.lat = Lattice(p.Nlx, p.Nly)
        if sigma is None:
            sigma, lam, r = seeded_config(p, self.lat, seed)
            self.lam = lam
            self.rng = r if rng is None else rng
        else:
            self.lam = np.ones(p.Lq)
            self.rng = Ranf(seed) if rng is None else rng
        self.sigma = np.array(sigma, dtype=np.float64)
        self.opk = OperatorKin(p, self.lat)
        self.opmu = OperatorMU(p)
        self.dtype = dtype
        N = p.Lq
        self.prop = Propagator(N, dtype)
        self.wr = WrapList(N, p.Nst, dtype)
        self.obs = ObserEqual(p, self.lat)
        self.obs_tau = ObserTau(p, self.lat)
        self.acc_num = 0.0
        self.acc_den = 0.0
        self.acc = 0.0
        self.record = record_decisions
        self.decisions = []
        self.ratios = []
        self.dyn_X = (np.zeros(3), np.zeros(3))
        # global update state (src/global_update.f90, src/main.f90:74-76)
        self.is_beta = True
        self.gacc = 0.0          # Acc_Kg%acc
        self.gsize = 0.0         # Wolff%size_cluster
        self.g_last = (0, 0)     # (accepted, proposed) of the last Global_sweep
        self.g_log = []          # (bond, size, log ratio space, fermion, accept) per move

    # ---- LocalK (src/localK.f90) ------------------------------------------
    def metro(self, ii: int, nt: int):
        """``LocalK_metro`` (src/localK.f90:45-173); nt 0-based."""
        G = self.prop.Gr
        sig = self.sigma
        s_old = sig[ii, nt]
        s_new = -s_old
        p1, p2 = self.lat.bond_list[ii]
        P = (p1, p2)
        Dl = self.opk.get_delta(ii, s_old, s_new)
        Gl = np.empty((2, 2), dtype=G.dtype)
        for nr in range(2):
            for nl in range(2):
                Gl[nl, nr] = (1.0 if nl == nr else 0.0) - G[P[nl], P[nr]]
        prod = np.empty((2, 2), dtype=G.dtype)
        for nr in range(2):
            for nl in range(2):
                m = Dl[nl, 0] * Gl[0, nr] + Dl[nl, 1] * Gl[1, nr]
                prod[nl, nr] = (1.0 if nl == nr else 0.0) + m
        det = prod[0, 0] * prod[1, 1] - prod[0, 1] * prod[1, 0]
        ratio_fermion = det * det
        ratio_boson = boson_ratio_local(self.p, self.lat, sig, ii, nt, s_new)
        ratio_re = float(np.real(ratio_fermion * ratio_boson))
        r = self.rng()
        accept = abs(ratio_re) > r
        self.acc_den += 1.0
        if self.record:
            self.decisions.append(bool(accept))
            self.ratios.append(ratio_re)
        if accept:
            self.acc_num += 1.0
            pinv = np.array([[prod[1, 1], -prod[0, 1]], [-prod[1, 0], prod[0, 0]]]) / det
            U = G[:, [p1, p2]].copy()
            V = np.empty((2, G.shape[0]), dtype=G.dtype)
            for no in range(2):
                V[no, :] = -Dl[no, 0] * G[p1, :] - Dl[no, 1] * G[p2, :]
                V[no, p1] += Dl[no, 0]
                V[no, p2] += Dl[no, 1]
            temp = U @ pinv
            diff = temp @ V
            self.prop.Gr = G - diff
            sig[ii, nt] = s_new
        return accept

    def prop_L(self, nt: int):
        """``LocalK_prop_L`` (src/localK.f90:347-373); nt 0-based."""
        for ii in range(2 * self.p.Lq - 1, -1, -1):
            self.metro(ii, nt)
        pr = self.prop
        self.opk.mmult_L(pr.Gr, self.sigma, nt, 1)
        self.opk.mmult_R(pr.Gr, self.sigma, nt, -1)
        self.opk.mmult_L(pr.UUL, self.sigma, nt, 1)

    def prop_R(self, nt: int):
        """``LocalK_prop_R`` (src/localK.f90:375-398); nt 0-based."""
        pr = self.prop
        self.opk.mmult_R(pr.Gr, self.sigma, nt, 1)
        self.opk.mmult_L(pr.Gr, self.sigma, nt, -1)
        for ii in range(2 * self.p.Lq):
            self.metro(ii, nt)
        self.opk.mmult_R(pr.UUR, self.sigma, nt, 1)

    # ---- multiply (src/multiply.f90) ---------------------------------------
    def propT_pre(self):
        self.prop.UUR = self.prop.UUR * self.opmu.expMU_P       # multiply.f90:65-77

    def propT_L(self):
        pr = self.prop                                           # multiply.f90:79-93
        pr.Gr = pr.Gr * self.opmu.expMU_P
        pr.Gr = pr.Gr * self.opmu.expMU_M
        pr.UUL = pr.UUL * self.opmu.expMU_P

    def propT_R(self):
        pr = self.prop                                           # multiply.f90:95-108
        pr.Gr = pr.Gr * self.opmu.expMU_P
        pr.Gr = pr.Gr * self.opmu.expMU_M
        pr.UUR = pr.UUR * self.opmu.expMU_P

    # ---- Wraps (src/stabilization.f90:374-476) -----------------------------
    def wrap_pre(self, nt: int):
        pr, wr, p = self.prop, self.wr, self.p
        st = nt // p.Nwrap
        if nt != 0:
            stab_UR(pr)
        wr.URlist[st], wr.VRlist[st], wr.DRlist[st] = pr.UUR, pr.VUR, pr.DUR
        if nt == p.Ltrot:
            pr.Gr = stab_green(pr, nt, p.Ltrot)

    def wrap_L(self, nt: int, flag=True):
        pr, wr, p = self.prop, self.wr, self.p
        st = nt // p.Nwrap
        pr.UUR, pr.VUR, pr.DUR = wr.URlist[st].copy(), wr.VRlist[st].copy(), wr.DRlist[st].copy()
        if nt == 0:
            wr.URlist[:] = 0.0
            wr.VRlist[:] = 0.0
            wr.DRlist[:] = 0.0
        if nt != p.Ltrot:
            stab_UL(pr)
            G = stab_green(pr, nt, p.Ltrot)
            dif = compare_mat(G, pr.Gr)
            pr.Xmaxm = max(pr.Xmaxm, dif)
            if flag:
                pr.Xmeanm += dif
            pr.Gr = G
        wr.ULlist[st], wr.VLlist[st], wr.DLlist[st] = pr.UUL.copy(), pr.VUL.copy(), pr.DUL.copy()

    def wrap_R(self, nt: int, flag=True):
        pr, wr, p = self.prop, self.wr, self.p
        st = nt // p.Nwrap
        pr.UUL, pr.VUL, pr.DUL = wr.ULlist[st].copy(), wr.VLlist[st].copy(), wr.DLlist[st].copy()
        if nt == p.Ltrot:
            wr.ULlist[:] = 0.0
            wr.VLlist[:] = 0.0
            wr.DLlist[:] = 0.0
        if nt != 0:
            stab_UR(pr)
            G = stab_green(pr, nt, p.Ltrot)
            dif = compare_mat(G, pr.Gr)
            pr.Xmaxm = max(pr.Xmaxm, dif)
            if flag:
                pr.Xmeanm += dif
            pr.Gr = G
        wr.URlist[st], wr.VRlist[st], wr.DRlist[st] = pr.UUR.copy(), pr.VUR.copy(), pr.DUR.copy()

    # ---- LocalSweep (src/local_sweep.f90) ----------------------------------
    def reset(self, toggle: bool):
        """``Local_sweep_reset`` (src/local_sweep.f90:56-71)."""
        self.acc_num = 0.0
        self.acc_den = 0.0
        self.obs.reset()
        if toggle:
            self.obs_tau.reset()
        if abs(self.p.h) <= ZERO:
            self.sigma[:, :] = self.sigma[:, :1]

    def pre(self):
        """``Local_sweep_pre`` (src/local_sweep.f90:87-104)."""
        p = self.p
        self.reset(False)
        self.wrap_pre(0)
        for nt in range(1, p.Ltrot + 1):
            if p.rt_scalar() > ZERO:
                self.opk.mmult_R(self.prop.UUR, self.sigma, nt - 1, 1)
            self.propT_pre()
            if nt % p.Nwrap == 0:
                self.wrap_pre(nt)

    def sweep_L(self):
        """``Local_sweep_L`` (src/local_sweep.f90:106-124)."""
        p = self.p
        for nt in range(p.Ltrot, 0, -1):
            if nt % p.Nwrap == 0:
                self.wrap_L(nt)
            self.obs.calc(self.prop.Gr, self.sigma, nt - 1)
            self.nobs += 1
            self.propT_L()
            self.prop_L(nt - 1)
        self.wrap_L(0)

    def sweep_R(self, toggle: bool):
        """``Local_sweep_R`` (src/local_sweep.f90:126-150)."""
        p = self.p
        if toggle:
            self.dyn_sweep()
            self.nobst += 1
        self.wrap_R(0)
        for nt in range(1, p.Ltrot + 1):
            self.prop_R(nt - 1)
            self.propT_R()
            if nt % p.Nwrap == 0:
                self.wrap_R(nt)
            self.obs.calc(self.prop.Gr, self.sigma, nt - 1)
            self.nobs += 1

    def sweep(self, toggle: bool = False, nsweep=None):
        """``Local_sweep`` (src/local_sweep.f90:152-195): one bin."""
        self.reset(toggle)
        self.nobs = 0
        self.nobst = 0
        for _ in range(self.p.Nsweep if nsweep is None else nsweep):
            if self.is_beta:
                self.sweep_L()
                self.sweep_R(toggle)
            else:
                self.sweep_R(toggle)
                self.sweep_L()
        self.obs.ave(self.nobs)
        if toggle:
            self.obs_tau.ave(self.nobst)
        if self.acc_den > 0.0:
            self.acc += self.acc_num / self.acc_den

    # ---- Boson-only warm-up (src/localK.f90:400-420, src/local_sweep.f90:73-85)
    def therm_sweep(self):
        """``Local_sweep_therm``: one pass of ``LocalK_therm`` over (nt, ii),
        Metropolis on the gauge weight alone; returns the accepted fraction
        (``Acc_Kt%ratio`` adds it to ``Acc_Kt%acc``)."""
        p = self.p
        if abs(p.h) <= ZERO:
            self.sigma[:, :] = self.sigma[:, :1]
        num = 0
        for nt in range(p.Ltrot):
            for ii in range(2 * p.Lq):
                s_new = -self.sigma[ii, nt]
                ratio = boson_ratio_local(p, self.lat, self.sigma, ii, nt, s_new)
                if ratio > self.rng():
                    self.sigma[ii, nt] = s_new
                    num += 1
        return num / float(2 * p.Lq * p.Ltrot)

    # ---- Global Wolff-in-tau move (src/global_update.f90, src/globalK.f90) --
    def nranf(self, N: int) -> int:
        """``nranf`` (src/calc_basic.f90:113-121): nint(ranf*N + 0.5),
        clamped to 1..N (1-based)."""
        x = self.rng() * float(N) + 0.5
        n = math.floor(x)
        if x - n >= 0.5:          # nint rounds half away from zero (x >= 0)
            n += 1
        return int(min(max(n, 1), N))

    def time_bond_prob(self) -> float:
        """``compute_time_bond_prob`` (src/global_update.f90:88-101)."""
        p = self.p
        if abs(p.h) > ZERO:
            ta = max(math.tanh(p.dtau * abs(p.h)), RATIO_EPS)
            gamma = -0.5 * math.log(ta)
            pt = 1.0 - math.exp(-2.0 * gamma)
        else:
            pt = 0.0
        return max(0.0, min(1.0, pt))

    def wolff_flip(self, sigma_new):
        """``Wolff_flip`` (src/global_update.f90:66-86): a time cluster on
        one bond, its plaquette log ratio, the flip applied to sigma_new.
        Returns (bond 0-based, cluster size, log ratio space)."""
        p = self.p
        L = p.Ltrot
        b = self.nranf(2 * p.Lq) - 1
        pt = self.time_bond_prob()
        # build_time_cluster (src/global_update.f90:103-131), 0-based tau
        mask = np.zeros(L, dtype=bool)
        q0 = self.nranf(L) - 1
        queue = [q0]
        mask[q0] = True
        head = 0
        while head < len(queue):
            cur = queue[head]
            head += 1
            for off in (-1, 1):
                nb = (cur + off) % L
                if mask[nb]:
                    continue
                if sigma_new[b, nb] == sigma_new[b, cur]:
                    # the reference evaluates ranf only when p_time > 0
                    if pt > 0.0 and self.rng() < pt:
                        queue.append(nb)
                        mask[nb] = True
        size = int(mask.sum())
        if size == 0:
            return b, 0, 0.0
        # compute_space_log_ratio / plaquette_log_ratio (src/global_update.f90:133-172)
        lrs = 0.0
        alpha = p.dtau * p.J
        if alpha != 0.0:
            bb = self.lat.bond_bonds
            for tau in range(L):
                if not mask[tau]:
                    continue
                for start in (1, 4):
                    prod = sigma_new[b, tau]
                    for k in range(3):
                        prod = prod * sigma_new[bb[b, start + k], tau]
                    lrs += -2.0 * alpha * prod
        sigma_new[b, mask] = -sigma_new[b, mask]   # apply_cluster_flip
        self._gmask = mask
        return b, size, lrs

    def ratio_k_fermion(self, sigma_new, ii: int, nt: int) -> float:
        """``ratioK_fermion`` (src/globalK.f90:15-113): |det Prod|^2 for the
        change sigma -> sigma_new at (ii, nt) and the G update; nt 0-based."""
        s_old = self.sigma[ii, nt]
        s_new = sigma_new[ii, nt]
        if s_new == s_old:
            return 1.0
        G = self.prop.Gr
        p1, p2 = self.lat.bond_list[ii]
        P = (p1, p2)
        Dl = self.opk.get_delta(ii, s_old, s_new)
        Gl = np.empty((2, 2), dtype=G.dtype)
        for nr in range(2):
            for nl in range(2):
                Gl[nl, nr] = (1.0 if nl == nr else 0.0) - G[P[nl], P[nr]]
        prod = np.empty((2, 2), dtype=G.dtype)
        for nr in range(2):
            for nl in range(2):
                m = Dl[nl, 0] * Gl[0, nr] + Dl[nl, 1] * Gl[1, nr]
                prod[nl, nr] = (1.0 if nl == nr else 0.0) + m
        det = prod[0, 0] * prod[1, 1] - prod[0, 1] * prod[1, 0]
        ratio = max(abs(det * det), RATIO_EPS)
        pinv = np.array([[prod[1, 1], -prod[0, 1]], [-prod[1, 0], prod[0, 0]]]) / det
        U = G[:, [p1, p2]].copy()
        V = np.empty((2, G.shape[0]), dtype=G.dtype)
        for no in range(2):
            V[no, :] = -Dl[no, 0] * G[p1, :] - Dl[no, 1] * G[p2, :]
            V[no, p1] += Dl[no, 0]
            V[no, p2] += Dl[no, 1]
        self.prop.Gr = G - (U @ pinv) @ V
        return float(ratio)

    def _global_move(self, left: bool):
        """``Global_sweep_L`` / ``Global_sweep_R`` (src/global_update.f90:228-318)
        on copies of the propagator and wrap lists."""
        p = self.p
        sigma_new = self.sigma.copy()
        b, size, lrs = self.wolff_flip(sigma_new)
        keep_prop, keep_wr = self.prop, self.wr
        self.prop, self.wr = keep_prop.copy(), _wrlist_copy(keep_wr)
        lrf = 0.0
        pr = self.prop
        if left:
            for nt in range(p.Ltrot, 0, -1):
                if nt % p.Nwrap == 0:
                    self.wrap_L(nt, flag=False)
                self.propT_L()
                for ii in range(2 * p.Lq - 1, -1, -1):   # GlobalK_prop_L (globalK.f90:115-133)
                    lrf += math.log(max(self.ratio_k_fermion(sigma_new, ii, nt - 1), RATIO_EPS))
                self.opk.mmult_L(pr.Gr, sigma_new, nt - 1, 1)
                self.opk.mmult_R(pr.Gr, sigma_new, nt - 1, -1)
                self.opk.mmult_L(pr.UUL, sigma_new, nt - 1, 1)
            self.wrap_L(0, flag=False)
        else:
            self.wrap_R(0, flag=False)
            for nt in range(1, p.Ltrot + 1):
                self.opk.mmult_R(pr.Gr, self.sigma, nt - 1, 1)   # GlobalK_prop_R (globalK.f90:135-153)
                self.opk.mmult_L(pr.Gr, self.sigma, nt - 1, -1)
                for ii in range(2 * p.Lq):
                    lrf += math.log(max(self.ratio_k_fermion(sigma_new, ii, nt - 1), RATIO_EPS))
                self.opk.mmult_R(pr.UUR, sigma_new, nt - 1, 1)
                self.propT_R()
                if nt % p.Nwrap == 0:
                    self.wrap_R(nt, flag=False)
        lrt = lrf + lrs
        r = self.rng()
        accept = min(0.0, lrt) >= math.log(max(r, RATIO_EPS))
        if accept:
            self.sigma = sigma_new
            self.is_beta = not left
        else:
            self.prop, self.wr = keep_prop, keep_wr
        self.g_log.append((b, size, lrs, lrf, bool(accept)))
        return accept, size

    def global_sweep(self, nglobal: int):
        """``Global_sweep`` (src/global_update.f90:320-337): Nglobal Wolff
        moves, each followed by a trial half-sweep in the current direction."""
        num = 0
        size = 0.0
        for _ in range(nglobal):
            acc, sz = self._global_move(self.is_beta)
            num += int(acc)
            size += float(sz)
        self.g_last = (num, nglobal)
        if nglobal > 0:
            self.gacc += num / nglobal
            self.gsize += size / nglobal

    # ---- Dynamics (src/dynamics.f90) ---------------------------------------
    def dyn_sweep(self):
        """``Dyn_reset`` + ``Dyn_sweep_R`` (src/dynamics.f90:41-62)."""
        p = self.p
        pd = self.prop.copy()
        pg = PropGreen(self.prop.Gr)
        pg.Xmaxm, pg.Xmeanm = self.dyn_X
        for nt in range(1, p.Ltrot + 1):
            self.obs_tau.calc(pg, self.sigma, nt - 1)
            if p.rt_scalar() > ZERO:
                self.opk.mmult_R(pg.Grt0, self.sigma, nt - 1, 1)        # multiply.f90:43-63
                self.opk.mmult_L(pg.Gr0t, self.sigma, nt - 1, -1)
                self.opk.mmult_R(pg.Grtt, self.sigma, nt - 1, 1)
                self.opk.mmult_L(pg.Grtt, self.sigma, nt - 1, -1)
                self.opk.mmult_R(pd.UUR, self.sigma, nt - 1, 1)
            eP, eM = self.opmu.expMU_P, self.opmu.expMU_M               # multiply.f90:110-130
            pg.Grt0 = pg.Grt0 * eP
            pg.Gr0t = pg.Gr0t * eM
            pg.Grtt = pg.Grtt * eP
            pg.Grtt = pg.Grtt * eM
            pd.UUR = pd.UUR * eP
            if nt % p.Nwrap == 0:
                self.wrap_tau(pd, pg, nt)
        self.dyn_X = (pg.Xmaxm, pg.Xmeanm)
        self.last_propgreen = pg

    def wrap_tau(self, pd: Propagator, pg: PropGreen, nt: int):
        """``Wrap_tau`` (src/stabilization.f90:478-514)."""
        st = nt // self.p.Nwrap
        wr = self.wr
        pd.UUL, pd.VUL, pd.DUL = wr.ULlist[st].copy(), wr.VLlist[st].copy(), wr.DLlist[st].copy()
        stab_UR(pd)
        g00, g0t, gt0, gtt = stab_green_big(pd)
        for k, (new, old) in enumerate(((g0t, pg.Gr0t), (gt0, pg.Grt0), (gtt, pg.Grtt))):
            dif = compare_mat(new, old)
            pg.Xmaxm[k] = max(pg.Xmaxm[k], dif)
            pg.Xmeanm[k] += dif
        pg.Gr00, pg.Gr0t, pg.Grt0, pg.Grtt = g00, g0t, gt0, gtt


# --------------------------------------------------------------------------
# Log-det and its adjoint (no reference routine; checked by finite
# differences and by the exact mu identity)
# --------------------------------------------------------------------------
def logdet_one_sector(p: Params, sigma) -> float:
    """log|det(1 + B_Ltrot ... B_1)| for one spin sector at fixed sigma,
    computed through the reference's own UDV chain (``Local_sweep_pre``,
    src/local_sweep.f90:87-104) and the pivoted QR of ``stab_green``'s
    middle matrix (src/stabilization.f90:134-151):
    det(1+UR DR VR) = det(UR) det(M), M = UR^T + DR VR, |det UR| = 1."""
    c = Z2Chain(p, sigma=sigma, seed=1)
    c.pre()
    pr = c.prop
    M = _ct(pr.UUR) + pr.DUR[:, None] * pr.VUR
    qr, D, jpvt, tau = qdrp_decompose(M)
    return float(np.sum(np.log(D)))


def logdet_grad_oracle(p: Params, sigma):
    """Exact gradient of log|det(1+B)| wrt per-bond hopping t_b and mu.

    With B = prod_l e^{dtau mu} E1 E2 E3 E4 E4 E3 E2 E1 and
    dE_g/dt_b = E_g (alpha_b/t_b) sigma_b X_b for b in g, the derivative of
    one factor F is Tr[(I - G_F) dF F^{-1}] where G_F is the equal-time
    Green's function whose product starts right after F.  The chain is
    walked factor by factor (G <- F G F^{-1}), with G recomputed from the
    UDV stacks at every Nwrap boundary.  d/dmu = beta Tr(I - G(0)).
    """
    c = Z2Chain(p, sigma=sigma, seed=1)
    c.pre()
    # left chain stacks (sweep_L without proposals)
    pL = p.Ltrot
    lat, opk = c.lat, c.opk
    for nt in range(pL, 0, -1):
        if nt % p.Nwrap == 0:
            c.wrap_L(nt, flag=False)
        c.propT_L()
        pr = c.prop
        opk.mmult_L(pr.Gr, c.sigma, nt - 1, 1)
        opk.mmult_R(pr.Gr, c.sigma, nt - 1, -1)
        opk.mmult_L(pr.UUL, c.sigma, nt - 1, 1)
    c.wrap_L(0, flag=False)
    G0 = c.prop.Gr.copy()
    dmu = p.beta * float(np.trace(np.eye(p.Lq) - G0))
    rt = p.rt_bond()
    grad = np.zeros(2 * p.Lq)
    c.wrap_R(0, flag=False)
    for nt in range(1, pL + 1):
        G = c.prop.Gr
        for g in GROUP_ORDER:
            grp = lat.groups[g]
            p1 = lat.bond_list[grp, 0]
            p2 = lat.bond_list[grp, 1]
            s = c.sigma[grp, nt - 1]
            grad[grp] += 0.5 * p.dtau * s * (-(G[p1, p2] + G[p2, p1]))
            # G <- F G F^{-1}: rows by F (nflag=+1), columns by F^{-1}
            opk.process_group(G, g, c.sigma, nt - 1, 1)
            opk.process_group_L(G, g, c.sigma, nt - 1, -1)
        c.prop.Gr = G
        opk.mmult_R(c.prop.UUR, c.sigma, nt - 1, 1)
        c.propT_R()
        if nt % p.Nwrap == 0:
            c.wrap_R(nt, flag=False)
    logdet = logdet_one_sector(p, sigma)
    return logdet, grad, dmu
