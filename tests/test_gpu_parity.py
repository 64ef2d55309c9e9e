"""GPU parity: the CUDA library through its C ABI against the CPU oracle
(a restatement of the reference routines, oracle/z2_oracle.py) on the same
seeded inputs.

Tolerances: integer work (sigma, ranf state, accept/reject decisions) is
bit-exact; floating-point Green's functions, determinant ratios and
observables agree within 1e-10 relative (max-abs difference over max-abs
value), the bar the hot path is held to.
"""
import numpy as np
import pytest

from oracle import z2_oracle as zo
from z2_gauge_zfy_b200 import Chain, Z2Batch
from z2_gauge_zfy_b200.api import integrate_susc, integrate_susc_freq

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def oracle_params(ch: Chain):
    return zo.Params(RT=ch.RT if ch.rt_bond is None else ch.rt_bond, J=ch.J, h=ch.h,
                     mu=ch.mu, Q=ch.Q, Nlx=ch.Nlx, Nly=ch.Nly, Ltrot=ch.Ltrot, beta=ch.beta,
                     Nwrap=ch.Nwrap, absolute=ch.absolute)


C1 = Chain(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=4, Nly=4, Ltrot=40, beta=4.0, Nwrap=10, seed=12345)


def test_seeded_config_bit_exact():
    for absolute in (1, 2, 3, 4, 5):
        ch = Chain(**{**C1.__dict__, "absolute": absolute})
        with Z2Batch([ch]) as b:
            sig, iseed = b.get_config(0)
        p = oracle_params(ch)
        lat = zo.Lattice(p.Nlx, p.Nly)
        s_o, lam, rng = zo.seeded_config(p, lat, ch.seed)
        assert np.array_equal(sig, s_o), absolute
        assert iseed == rng.state, absolute


@pytest.mark.parametrize("Lx,Ly", [(4, 4), (6, 6), (8, 8), (12, 12), (4, 6), (6, 4)])
def test_mmult_parity(Lx, Ly):
    """B^nflag M and M B^nflag (mmult_R / mmult_L).  Square lattices take the
    fused line kernels, rectangular ones the pass-by-pass kernel."""
    ch = Chain(RT=1.0, Nlx=Lx, Nly=Ly, Ltrot=20, beta=2.0, Nwrap=10, seed=777)
    rng = np.random.default_rng(1)
    N = Lx * Ly
    with Z2Batch([ch]) as b:
        p = oracle_params(ch)
        lat = zo.Lattice(Lx, Ly)
        sig, _, _ = zo.seeded_config(p, lat, ch.seed)
        opk = zo.OperatorKin(p, lat)
        for nt in (1, 7, 20):
            for nflag in (1, -1):
                M = rng.standard_normal((N, N))
                gR = b.opk_mmult_R(0, M, nt, nflag)
                oR = M.copy()
                opk.mmult_R(oR, sig, nt - 1, nflag)
                assert rel(gR, oR) < 1e-14
                gL = b.opk_mmult_L(0, M, nt, nflag)
                oL = M.copy()
                opk.mmult_L(oL, sig, nt - 1, nflag)
                assert rel(gL, oL) < 1e-14


def _propagated_udv(ch, nslices=10):
    p = oracle_params(ch)
    c = zo.Z2Chain(p, seed=ch.seed)
    U = np.eye(p.Lq)
    for nt in range(nslices):
        c.opk.mmult_R(U, c.sigma, nt, 1)
    return c, U


@pytest.mark.parametrize("L", [4, 8, 12])
def test_stab_U_parity(L):
    ch = Chain(RT=1.0, Nlx=L, Nly=L, Ltrot=40, beta=4.0, Nwrap=10, seed=4242)
    c, U = _propagated_udv(ch)
    N = ch.N
    rng = np.random.default_rng(2)
    D = np.exp(rng.uniform(-3, 3, N))
    V = np.triu(rng.standard_normal((N, N))) + 3 * np.eye(N)
    with Z2Batch([ch]) as b:
        for left in (False, True):
            pr = zo.Propagator(N)
            if left:
                pr.UUL, pr.DUL, pr.VUL = U.T.copy(), D.copy(), V.copy()
                zo.stab_UL(pr)
                Ug, Dg, Vg = b.stab_UL(0, U.T.copy(), D, V)
                ref = (pr.VUL * pr.DUL[None, :]) @ pr.UUL
                got = (Vg * Dg[None, :]) @ Ug
                assert rel(Dg, pr.DUL) < RTOL
            else:
                pr.UUR, pr.DUR, pr.VUR = U.copy(), D.copy(), V.copy()
                zo.stab_UR(pr)
                Ug, Dg, Vg = b.stab_UR(0, U, D, V)
                ref = pr.UUR @ (pr.DUR[:, None] * pr.VUR)
                got = Ug @ (Dg[:, None] * Vg)
                assert rel(Dg, pr.DUR) < RTOL
            assert rel(got, ref) < RTOL
            assert np.max(np.abs(Ug.T @ Ug - np.eye(N))) < 1e-13


@pytest.mark.parametrize("nt", [0, 10, 20, 30, 40])
def test_stab_green_parity(nt):
    ch = C1
    p = oracle_params(ch)
    c = zo.Z2Chain(p, seed=ch.seed)
    c.pre()
    pr = c.prop
    # UR chain from pre, a non-trivial UL chain from the reversed stack
    st = min(nt // p.Nwrap, p.Nst)
    UR, DR, VR = c.wr.URlist[st], c.wr.DRlist[st], c.wr.VRlist[st]
    rng = np.random.default_rng(3)
    UL, _ = np.linalg.qr(rng.standard_normal((p.Lq, p.Lq)))
    DL = np.exp(rng.uniform(-4, 4, p.Lq))
    VL = np.triu(rng.standard_normal((p.Lq, p.Lq))) + 3 * np.eye(p.Lq)
    t = zo.Propagator(p.Lq)
    t.UUR, t.DUR, t.VUR, t.UUL, t.DUL, t.VUL = UR, DR, VR, UL, DL, VL
    Go = zo.stab_green(t, nt, p.Ltrot)
    with Z2Batch([ch]) as b:
        Gg = b.stab_green(0, UR, DR, VR, UL, DL, VL, nt)
    assert rel(Gg, Go) < RTOL


def test_stab_green_big_parity():
    ch = C1
    p = oracle_params(ch)
    c = zo.Z2Chain(p, seed=ch.seed)
    c.pre()
    UR, DR, VR = c.wr.URlist[2], c.wr.DRlist[2], c.wr.VRlist[2]
    rng = np.random.default_rng(5)
    UL, _ = np.linalg.qr(rng.standard_normal((p.Lq, p.Lq)))
    DL = np.exp(rng.uniform(-2, 2, p.Lq))
    VL = np.triu(rng.standard_normal((p.Lq, p.Lq))) + 3 * np.eye(p.Lq)
    t = zo.Propagator(p.Lq)
    t.UUR, t.DUR, t.VUR, t.UUL, t.DUL, t.VUL = UR, DR, VR, UL, DL, VL
    ref = zo.stab_green_big(t)
    with Z2Batch([ch]) as b:
        got = b.stab_green_big(0, UR, DR, VR, UL, DL, VL)
    for g, o in zip(got, ref):
        assert rel(g, o) < 1e-9


def test_pre_parity():
    p = oracle_params(C1)
    c = zo.Z2Chain(p, seed=C1.seed)
    c.pre()
    with Z2Batch([C1]) as b:
        b.pre()
        G = b.green(0)
    assert rel(G, c.prop.Gr) < RTOL


def _run_pair(ch, nbins=1, toggle=False, nsweep=1, replay=None, delay_k=0):
    p = oracle_params(ch)
    rng = zo.ReplayStream(replay) if replay is not None else None
    c = zo.Z2Chain(p, seed=ch.seed, rng=rng, record_decisions=True)
    c.pre()
    with Z2Batch([ch], record=True, delay_k=delay_k, tau=toggle) as b:
        if replay is not None:
            b.set_replay(0, replay)
        b.pre()
        res = []
        for _ in range(nbins):
            c.decisions, c.ratios = [], []
            c.sweep(toggle=toggle, nsweep=nsweep)
            b.sweep(nsweep, toggle)
            res.append((b.green(0), b.obs_equal(0), b.stats(0), b.decisions(0),
                        b.obs_tau(0) if toggle else None, b.get_config(0),
                        b.obs_tau_k(0) if toggle else None))
    return c, res


def _decisions_oracle(c, L, nb):
    d = np.array(c.decisions[-2 * L * nb:], dtype=np.uint8).reshape(2, L, nb)
    r = np.array(c.ratios[-2 * L * nb:]).reshape(2, L, nb)
    # the oracle records the L half-sweep in bond order 2N..1 and slices Ltrot..1
    d0 = d[0][::-1, ::-1]
    r0 = r[0][::-1, ::-1]
    return np.stack([d0, d[1]]), np.stack([r0, r[1]])


def test_sweep_parity_c1():
    ch = C1
    c, res = _run_pair(ch, nbins=2)
    G, obs, st, (dec, rat), _, (sig, iseed), _ = res[-1]
    dec_o, rat_o = _decisions_oracle(c, ch.Ltrot, 2 * ch.N)
    assert np.array_equal(dec, dec_o)
    assert rel(rat, rat_o) < RTOL
    assert np.array_equal(sig, c.sigma)
    assert iseed == c.rng.state
    assert rel(G, c.prop.Gr) < RTOL
    for k, v in c.obs.as_dict().items():
        assert abs(obs[k] - v) <= RTOL * max(abs(v), 1.0), k
    assert abs(st["Xmaxm"] - c.prop.Xmaxm) <= 1e-9 * max(c.prop.Xmaxm, 1e-3)


@pytest.mark.parametrize("Lx,Ly", [(4, 6), (6, 4)])
def test_sweep_parity_rectangular(Lx, Ly):
    """Lx != Ly: the pass-by-pass checkerboard kernel (the fused line kernels
    only take square lattices); decisions bit-exact, G within tolerance."""
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=Lx, Nly=Ly, Ltrot=20, beta=2.0, Nwrap=5,
               seed=2024)
    c, res = _run_pair(ch, nbins=1)
    G, obs, st, (dec, rat), _, (sig, iseed), _ = res[-1]
    dec_o, rat_o = _decisions_oracle(c, ch.Ltrot, 2 * ch.N)
    assert np.array_equal(dec, dec_o)
    assert np.array_equal(sig, c.sigma)
    assert rel(G, c.prop.Gr) < RTOL
    for k, v in c.obs.as_dict().items():
        assert abs(obs[k] - v) <= RTOL * max(abs(v), 1.0), k


def test_sweep_parity_mu_replay_all_accept():
    """Every proposal accepted (replayed uniforms 0), mu != 0: stresses the
    delayed-update queue and the mu scaling."""
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.2, Nlx=4, Nly=4, Ltrot=20, beta=2.0, Nwrap=5,
               seed=99)
    n = 2 * 2 * ch.N * ch.Ltrot
    c, res = _run_pair(ch, replay=np.zeros(n))
    G, obs, st, (dec, rat), _, (sig, _), _ = res[-1]
    dec_o, rat_o = _decisions_oracle(c, ch.Ltrot, 2 * ch.N)
    assert np.array_equal(dec, dec_o)
    assert rel(G, c.prop.Gr) < RTOL
    assert np.array_equal(sig, c.sigma)


def test_sweep_parity_tau():
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.1, Nlx=4, Nly=4, Ltrot=20, beta=2.0, Nwrap=5,
               seed=2024)
    c, res = _run_pair(ch, toggle=True)
    G, obs, st, _, otau, _, otau_k = res[-1]
    assert rel(G, c.prop.Gr) < RTOL
    lat = zo.Lattice(ch.Nlx, ch.Nly)
    dtau = ch.beta / ch.Ltrot
    for q, k in enumerate(zo.TAU_NAMES):
        ref = np.real(c.obs_tau.arr[k])
        assert rel(otau[k], ref) < 1e-9, k
        # momentum space (Fourier_R_to_K of the output layer) on the GPU
        gk_ref = zo.fourier_r_to_k(c.obs_tau.arr[k], lat)
        assert np.max(np.abs(otau_k[k] - gk_ref)) <= 1e-9 * max(np.max(np.abs(gk_ref)), 1e-12), k
        s_ref = zo.integrate_susc(gk_ref, dtau)
        assert np.max(np.abs(integrate_susc(otau_k[k], dtau) - s_ref)) <= \
            1e-9 * max(np.max(np.abs(s_ref)), 1e-12), k
    w_ref = zo.integrate_susc_freq(zo.fourier_r_to_k(c.obs_tau.arr["curxx"], lat), dtau)
    w = integrate_susc_freq(otau_k["curxx"], dtau)
    assert np.max(np.abs(w - w_ref)) <= 1e-9 * max(np.max(np.abs(w_ref)), 1e-12)


def test_logdet_grad_parity():
    L = 4
    N = L * L
    rng = np.random.default_rng(11)
    rt = 1.0 + 0.05 * rng.standard_normal(2 * N)
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.1, Nlx=L, Nly=L, Ltrot=20, beta=2.0, Nwrap=5,
               seed=31, rt_bond=rt)
    p = oracle_params(ch)
    lat = zo.Lattice(L, L)
    sig, _, _ = zo.seeded_config(p, lat, ch.seed)
    ld_o, g_o, dmu_o = zo.logdet_grad_oracle(p, sig)
    with Z2Batch([ch]) as b:
        ld, g, dmu = b.logdet_grad(0)
    assert abs(ld - ld_o) <= 1e-10 * abs(ld_o)
    assert rel(g, g_o) < 1e-9
    assert abs(dmu - dmu_o) <= 1e-10 * abs(dmu_o)


def test_sweep_parity_L16_global_G():
    """N = 256: G does not fit in shared memory and lives in global memory
    (same kernels through generic pointers)."""
    ch = Chain(RT=1.0, J=0.5, h=0.6, mu=0.0, Nlx=16, Nly=16, Ltrot=16, beta=0.8, Nwrap=8,
               seed=4321)
    c, res = _run_pair(ch)
    G, obs, st, (dec, rat), _, (sig, iseed), _ = res[-1]
    dec_o, _ = _decisions_oracle(c, ch.Ltrot, 2 * ch.N)
    assert np.array_equal(dec, dec_o)
    assert np.array_equal(sig, c.sigma) and iseed == c.rng.state
    assert rel(G, c.prop.Gr) < RTOL


def test_graph_replay_and_delay_rank_identical_decisions():
    chains = [Chain(RT=1.0, J=0.5, h=0.5, Nlx=6, Nly=6, Ltrot=20, beta=2.0, Nwrap=10, seed=s)
              for s in (11, 12)]
    outs = []
    for kw in (dict(), dict(graph=True), dict(delay_k_chain=[4, 32])):
        with Z2Batch(chains, record=True, **kw) as b:
            b.pre()
            for _ in range(3):
                b.sweep(1, False)
            outs.append([(b.green(i), b.decisions(i)[0], b.get_config(i)[0]) for i in range(2)])
    for i in range(2):
        g0, d0, s0 = outs[0][i]
        g1, d1, s1 = outs[1][i]
        assert np.array_equal(g0, g1) and np.array_equal(d0, d1) and np.array_equal(s0, s1)
        g2, d2, s2 = outs[2][i]
        assert np.array_equal(d0, d2) and np.array_equal(s0, s2)
        assert rel(g2, g0) < RTOL


def test_delay_autotuner():
    """z2_tune_delay gives one rank per lattice size from its candidate list,
    and a batch built with the tuned ranks makes the same decisions."""
    from z2_gauge_zfy_b200 import tune_delay
    chains = [Chain(RT=1.0, J=0.5, h=0.5, Nlx=L, Nly=L, Ltrot=20, beta=2.0, Nwrap=10, seed=s)
              for L, s in ((4, 21), (6, 22), (4, 23), (6, 24))]
    k = tune_delay(chains)
    assert k.shape == (4,)
    assert set(k.tolist()) <= {4, 6, 8, 12, 16, 24, 32, 48, 64}
    assert k[0] == k[2] and k[1] == k[3]
    outs = []
    for kw in (dict(), dict(delay_k="auto")):
        with Z2Batch(chains, record=True, **kw) as b:
            b.pre()
            b.sweep(2, False)
            outs.append([(b.green(i), b.decisions(i)[0]) for i in range(4)])
    for (g0, d0), (g1, d1) in zip(*outs):
        assert np.array_equal(d0, d1)
        assert rel(g1, g0) < RTOL


def test_flush_shapes_identical_bits():
    """Every tile shape of the rank-2k flush forms each element of G with the
    same k chunks, so a batch run with any valid shape makes the same
    decisions and leaves the same G, to the bit (N = 144 admits all seven
    explicit shapes, N = 64 four, N = 36 the two bounded ones)."""
    from z2_gauge_zfy_b200 import FLUSH_SHAPES
    chains = [Chain(RT=1.0, J=0.5, h=0.6, Nlx=L, Nly=L, Ltrot=20, beta=2.0, Nwrap=10, seed=70 + L)
              for L in (12, 8, 6)]
    ok = {144: set(range(8)), 64: {0, 1, 2, 3, 4, 6}, 36: {0, 1, 2}}
    ref = None
    for shape in sorted(FLUSH_SHAPES):
        sh = [shape if shape in ok[c.N] else 0 for c in chains]
        with Z2Batch(chains, record=True, delay_k=8, flush_shape_chain=sh) as b:
            b.pre()
            b.sweep(1, False)
            out = [(b.green(i), b.decisions(i)[0]) for i in range(len(chains))]
        if ref is None:
            ref = out
            continue
        for (g0, d0), (g1, d1) in zip(ref, out):
            assert np.array_equal(d0, d1), shape
            assert np.array_equal(g0, g1), shape


def test_tuner_shapes_valid_and_repeatable():
    """z2_tune picks one (rank, shape) per lattice size, valid for that size,
    and two consecutive calls pick the same."""
    from z2_gauge_zfy_b200 import tune
    chains = [Chain(RT=1.0, J=0.5, h=0.5, Nlx=L, Nly=L, Ltrot=40, beta=4.0, Nwrap=10, seed=s)
              for L, s in ((6, 1), (8, 2), (12, 3), (6, 4), (12, 5))]
    k1, s1 = tune(chains)
    k2, s2 = tune(chains)
    assert np.array_equal(k1, k2) and np.array_equal(s1, s2), (k1, s1, k2, s2)
    assert k1[0] == k1[3] and s1[0] == s1[3] and k1[2] == k1[4] and s1[2] == s1[4]
    ok = {36: {0, 1, 2}, 64: {0, 1, 2, 3, 4, 6}, 144: set(range(8))}
    for c, k, s in zip(chains, k1, s1):
        assert int(s) in ok[c.N], (c.N, s)
        assert k in (4, 6, 8, 12, 16, 24, 32, 48, 64)


def test_obs_equal_all_matches_per_chain_readback():
    """z2_get_obs_equal_all (one gather, one copy) returns exactly what
    z2_get_obs_equal returns chain by chain."""
    chains = [Chain(RT=1.0, J=0.5, h=0.5, Nlx=L, Nly=L, Ltrot=20, beta=2.0, Nwrap=10, seed=s)
              for L, s in ((4, 1), (6, 2), (8, 3))]
    with Z2Batch(chains) as b:
        b.pre()
        b.sweep(1, False)
        allv = b.obs_equal_all()
        per = np.array([list(b.obs_equal(i).values()) for i in range(len(chains))])
    assert allv.shape == (3, 7) and np.array_equal(allv, per)
