"""Parity at production lattice sizes for the time-displaced path and the
adjoint, through the C ABI against the oracle (oracle/z2_oracle.py).

- stab_green_big (src/stabilization.f90:202-264) at N = 144 and N = 256 on the
  UDV stacks of real chains: UR, DR, VR from Local_sweep_pre's right chain and
  UL, DL, VL from a left half-sweep's stack at the same stabilization point,
  the pair Wrap_tau hands to stab_green_big (src/stabilization.f90:478-514).
- a toggle bin at N = 144 and N = 256 (sweep_L, sweep_R and Dyn%sweep_R,
  src/dynamics.f90:41-62; propgrK_R, src/multiply.f90:43-63; the seven
  Obs_tau correlators, src/obser_tau.f90:56-133): decisions bit-identical,
  G, the correlators and their momentum-space transforms within 1e-10.
- the adjoint of log det at the full adjoint configuration (L = 12, beta = 12,
  120 slices, per-bond hopping 1 + 0.05 N(0,1), mu = 0.1) against the
  oracle's exact gradient.

Tolerances are relative: max-abs difference over max-abs value.
"""
import numpy as np
import pytest

from oracle import z2_oracle as zo
from z2_gauge_zfy_b200 import Chain, Z2Batch

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _params(ch):
    return zo.Params(RT=ch.RT if ch.rt_bond is None else ch.rt_bond, J=ch.J, h=ch.h, mu=ch.mu,
                     Q=ch.Q, Nlx=ch.Nlx, Nly=ch.Nly, Ltrot=ch.Ltrot, beta=ch.beta,
                     Nwrap=ch.Nwrap, absolute=ch.absolute)


@pytest.mark.parametrize("L,Ltrot,Nwrap,st", [(12, 40, 10, 2), (16, 16, 8, 1)])
def test_stab_green_big_at_size(L, Ltrot, Nwrap, st):
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=L, Nly=L, Ltrot=Ltrot, beta=0.1 * Ltrot,
               Nwrap=Nwrap, seed=3000 + L)
    c = zo.Z2Chain(_params(ch), seed=ch.seed)
    c.pre()
    wr = c.wr
    UR, DR, VR = wr.URlist[st].copy(), wr.DRlist[st].copy(), wr.VRlist[st].copy()
    c.nobs = 0
    c.sweep_L()
    UL, DL, VL = wr.ULlist[st].copy(), wr.DLlist[st].copy(), wr.VLlist[st].copy()
    t = zo.Propagator(ch.N)
    t.UUR, t.DUR, t.VUR, t.UUL, t.DUL, t.VUL = UR, DR, VR, UL, DL, VL
    ref = zo.stab_green_big(t)
    with Z2Batch([ch]) as b:
        got = b.stab_green_big(0, UR, DR, VR, UL, DL, VL)
    errs = [rel(g, o) for g, o in zip(got, ref)]
    print(f"N={ch.N}: G00, G0t, Gt0, Gtt rel errors {errs}")
    assert max(errs) < RTOL, errs


@pytest.mark.parametrize("L,Ltrot,Nwrap", [(12, 20, 10), (16, 16, 8)])
def test_tau_bin_at_size(L, Ltrot, Nwrap):
    """N = 144 (G in shared memory) and N = 256 (G in HBM, the large batched
    configuration's lattice and Nwrap), a whole toggle bin against the oracle."""
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.1, Nlx=L, Nly=L, Ltrot=Ltrot, beta=0.1 * Ltrot,
               Nwrap=Nwrap, seed=1441 + L)
    p = _params(ch)
    c = zo.Z2Chain(p, seed=ch.seed, record_decisions=True)
    c.pre()
    c.decisions, c.ratios = [], []
    c.sweep(toggle=True)
    with Z2Batch([ch], record=True, tau=True) as b:
        b.pre()
        b.sweep(1, True)
        G, otau, otau_k, st = b.green(0), b.obs_tau(0), b.obs_tau_k(0), b.stats(0)
        dec, _ = b.decisions(0)
        sig, iseed = b.get_config(0)
    nb, Lt = 2 * ch.N, ch.Ltrot
    d = np.array(c.decisions, dtype=np.uint8).reshape(2, Lt, nb)
    assert np.array_equal(dec, np.stack([d[0][::-1, ::-1], d[1]]))
    assert np.array_equal(sig, c.sigma) and iseed == c.rng.state
    assert rel(G, c.prop.Gr) < RTOL
    lat = zo.Lattice(ch.Nlx, ch.Nly)
    worst = 0.0
    for k in zo.TAU_NAMES:
        ref = np.real(c.obs_tau.arr[k])
        e = rel(otau[k], ref)
        ek = rel(otau_k[k], zo.fourier_r_to_k(c.obs_tau.arr[k], lat))
        worst = max(worst, e, ek)
        assert e < RTOL, (k, e)
        assert ek < RTOL, (k, ek)
    # drift of the time-displaced chain (Xmaxm(1:3) of PropGreen)
    for q in range(3):
        xo = c.dyn_X[0][q]
        assert abs(st[f"Xmaxm_tau{q}"] - xo) <= 1e-10 + 1e-6 * xo, (q, st[f"Xmaxm_tau{q}"], xo)
    print(f"tau bin N={ch.N}: worst correlator rel error {worst:.2e}")


def test_logdet_grad_at_adjoint_size():
    L = 12
    N = L * L
    rng = np.random.default_rng(4)
    rt = 1.0 + 0.05 * rng.standard_normal(2 * N)
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.1, Nlx=L, Nly=L, Ltrot=120, beta=12.0, Nwrap=10,
               seed=20250, rt_bond=rt)
    p = _params(ch)
    sig, _, _ = zo.seeded_config(p, zo.Lattice(L, L), ch.seed)
    ld_o, g_o, dmu_o = zo.logdet_grad_oracle(p, sig)
    with Z2Batch([ch]) as b:
        ld, g, dmu = b.logdet_grad(0)
    print(f"logdet rel {abs(ld - ld_o) / abs(ld_o):.2e}, grad rel {rel(g, g_o):.2e}, "
          f"dmu rel {abs(dmu - dmu_o) / abs(dmu_o):.2e}")
    assert abs(ld - ld_o) <= 1e-10 * abs(ld_o)
    assert rel(g, g_o) < 1e-9
    assert abs(dmu - dmu_o) <= 1e-10 * abs(dmu_o)
