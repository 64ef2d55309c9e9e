"""The module-level mirrors through the C ABI, against the oracle's routines of
the same names (oracle/z2_oracle.py, a restatement of the reference).

A driver that replaces the reference's modules one at a time calls these
entry points in the reference's own order.  Here the tests do exactly that:
Local_sweep_pre (src/local_sweep.f90:87-104) and one whole bin with the
time-displaced pass (Local_sweep_L / _R, src/local_sweep.f90:106-150;
Dyn_sweep_R, src/dynamics.f90:50-62) are driven procedure by procedure
(propK_*, propT_*, propgr*, Wrap_*, Dyn_reset, LocalK_prop_L/R,
Obs_equal%calc/ave, Obs_tau%calc/ave) and compared with the oracle and with
the library's own whole-bin z2_sweep.  The multiply procedures are also
checked one by one on random matrices.

Tolerances: decisions, links and ranf state bit-exact; matrices and
observables within 1e-10 relative (max-abs difference over max-abs value).
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


CH = Chain(RT=1.0, J=0.5, h=0.5, mu=0.1, Nlx=6, Nly=6, Ltrot=20, beta=2.0, Nwrap=5, seed=606)


def _oracle(ch, record=False):
    p = zo.Params(RT=ch.RT, J=ch.J, h=ch.h, mu=ch.mu, Q=ch.Q, Nlx=ch.Nlx, Nly=ch.Nly,
                  Ltrot=ch.Ltrot, beta=ch.beta, Nwrap=ch.Nwrap, absolute=ch.absolute)
    return zo.Z2Chain(p, seed=ch.seed, record_decisions=record)


def _pre_by_modules(b, ch):
    """Local_sweep_pre: reset, Propagator = identity, Wrap_pre(0), then
    propK_pre / propT_pre per slice and Wrap_pre at every stabilization."""
    N = ch.N
    eye = np.eye(N)
    b.sweep_reset(0, False)
    b.set_prop(0, G=eye, UR=eye, DR=np.ones(N), VR=eye, UL=eye, DL=np.ones(N), VL=eye)
    b.wrap_pre(0, 0)
    for nt in range(1, ch.Ltrot + 1):
        b.propK_pre(0, nt)
        b.propT_pre(0)
        if nt % ch.Nwrap == 0:
            b.wrap_pre(0, nt)


def _bin_by_modules(b, ch):
    """One bin with toggle (is_beta: sweep_L then sweep_R with the
    time-displaced pass), procedure by procedure."""
    L, nw = ch.Ltrot, ch.Nwrap
    b.sweep_reset(0, True)
    nobs = 0
    for nt in range(L, 0, -1):                   # Local_sweep_L
        if nt % nw == 0:
            b.wrap_L(0, nt, True)
        b.obs_equal_calc(0, nt)
        nobs += 1
        b.propT_L(0)
        b.prop_slice_L(0, nt)
    b.wrap_L(0, 0, True)
    b.dyn_reset(0)                               # Dyn%reset + Dyn%sweep_R
    for nt in range(1, L + 1):
        b.obs_tau_calc(0, nt)
        b.propgrK_R(0, nt)
        b.propgrT_R(0)
        if nt % nw == 0:
            b.wrap_tau(0, nt)
    b.wrap_R(0, 0, True)                         # Local_sweep_R
    for nt in range(1, L + 1):
        b.prop_slice_R(0, nt)
        b.propT_R(0)
        if nt % nw == 0:
            b.wrap_R(0, nt, True)
        b.obs_equal_calc(0, nt)
        nobs += 1
    b.obs_equal_ave(0, nobs)
    b.obs_tau_ave(0, 1)


def test_pre_by_modules_matches_oracle_and_z2_pre():
    c = _oracle(CH)
    c.pre()
    with Z2Batch([CH], tau=True) as a, Z2Batch([CH], tau=True) as b:
        _pre_by_modules(a, CH)
        b.pre()
        pa, pb = a.get_prop(0), b.get_prop(0)
    assert rel(pa["G"], c.prop.Gr) < RTOL
    assert rel(pa["G"], pb["G"]) < 1e-13
    # the UDV factors of the right chain at the last stabilization
    got = pa["UR"] @ (pa["DR"][:, None] * pa["VR"])
    ref = c.prop.UUR @ (c.prop.DUR[:, None] * c.prop.VUR)
    assert rel(got, ref) < RTOL


def test_bin_by_modules_matches_oracle_and_z2_sweep():
    c = _oracle(CH, record=True)
    c.pre()
    c.decisions, c.ratios = [], []
    c.sweep(toggle=True)
    with Z2Batch([CH], tau=True, record=True) as a, Z2Batch([CH], tau=True, record=True) as b:
        a.pre()
        _bin_by_modules(a, CH)
        b.pre()
        b.sweep(1, True)
        out = []
        for h in (a, b):
            out.append(dict(G=h.green(0), obs=h.obs_equal(0), tau=h.obs_tau(0),
                            dec=h.decisions(0)[0], cfg=h.get_config(0), st=h.stats(0),
                            gr=h.get_propgr(0)))
    ga, gb = out
    nb, L = 2 * CH.N, CH.Ltrot
    d = np.array(c.decisions, dtype=np.uint8).reshape(2, L, nb)
    assert np.array_equal(ga["dec"], np.stack([d[0][::-1, ::-1], d[1]]))
    assert np.array_equal(ga["dec"], gb["dec"])
    assert np.array_equal(ga["cfg"][0], c.sigma) and ga["cfg"][1] == c.rng.state
    assert rel(ga["G"], c.prop.Gr) < RTOL
    assert rel(ga["G"], gb["G"]) < 1e-12
    for k, v in c.obs.as_dict().items():
        assert abs(ga["obs"][k] - v) <= RTOL * max(abs(v), 1.0), k
        assert abs(ga["obs"][k] - gb["obs"][k]) <= 1e-12 * max(abs(v), 1.0), k
    for k in zo.TAU_NAMES:
        assert rel(ga["tau"][k], np.real(c.obs_tau.arr[k])) < RTOL, k
    pg = c.last_propgreen
    for name, ref in (("G00", pg.Gr00), ("G0t", pg.Gr0t), ("Gt0", pg.Grt0), ("Gtt", pg.Grtt)):
        assert rel(ga["gr"][name], ref) < RTOL, name
    assert abs(ga["st"]["Xmaxm"] - c.prop.Xmaxm) <= 1e-9 * max(c.prop.Xmaxm, 1e-3)


def test_multiply_procedures_on_random_state():
    """propK_L / propK_R / propT_L / propT_R / propgrK_R / propgrT_R on a
    random Propagator, one call each, against the oracle's checkerboard
    operator (OperatorKin%mmult_R/L, src/operator_kin.f90:61-145) and mu
    factors (src/multiply.f90:65-130)."""
    rng = np.random.default_rng(8)
    N, nt = CH.N, 7
    c = _oracle(CH)
    opk, sig = c.opk, c.sigma
    eP, eM = np.exp(CH.beta / CH.Ltrot * CH.mu), np.exp(-CH.beta / CH.Ltrot * CH.mu)
    G0, UR0, UL0 = rng.standard_normal((3, N, N))
    with Z2Batch([CH], tau=True) as b:
        b.set_prop(0, G=G0, UR=UR0, UL=UL0)
        b.propK_R(0, nt)
        p = b.get_prop(0)
        G, UR = G0.copy(), UR0.copy()
        opk.mmult_R(G, sig, nt - 1, 1)
        opk.mmult_L(G, sig, nt - 1, -1)
        opk.mmult_R(UR, sig, nt - 1, 1)
        assert rel(p["G"], G) < 1e-13 and rel(p["UR"], UR) < 1e-13
        b.propT_R(0)
        p = b.get_prop(0)
        assert rel(p["G"], G * eP * eM) < 1e-14 and rel(p["UR"], UR * eP) < 1e-14
        b.set_prop(0, G=G0, UL=UL0)
        b.propK_L(0, nt)
        b.propT_L(0)
        p = b.get_prop(0)
        G, UL = G0.copy(), UL0.copy()
        opk.mmult_L(G, sig, nt - 1, 1)
        opk.mmult_R(G, sig, nt - 1, -1)
        opk.mmult_L(UL, sig, nt - 1, 1)
        assert rel(p["G"], G * eP * eM) < 1e-13 and rel(p["UL"], UL * eP) < 1e-13
        # time-displaced: Dyn_reset from G0, then propgrK_R and propgrT_R
        b.set_prop(0, G=G0)
        b.dyn_reset(0)
        b.propgrK_R(0, nt)
        b.propgrT_R(0)
        gr = b.get_propgr(0)
        gt0, g0t, gtt = G0.copy(), -(np.eye(N) - G0), G0.copy()
        opk.mmult_R(gt0, sig, nt - 1, 1)
        opk.mmult_L(g0t, sig, nt - 1, -1)
        opk.mmult_R(gtt, sig, nt - 1, 1)
        opk.mmult_L(gtt, sig, nt - 1, -1)
        assert rel(gr["Gt0"], gt0 * eP) < 1e-13
        assert rel(gr["G0t"], g0t * eM) < 1e-13
        assert rel(gr["Gtt"], gtt * eP * eM) < 1e-13
        assert rel(gr["G00"], G0) == 0.0
