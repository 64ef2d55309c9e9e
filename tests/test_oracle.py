"""Known-answer tests that pin the CPU oracle (oracle/z2_oracle.py).

The reference (Fortran + MPI + LAPACK) cannot be compiled in this image; its
one recorded run pins the oracle in tests/test_oracle_testrun.py.  Beyond
that run the oracle is pinned by:
  * the ranf recursion against its closed form,
  * lattice-table invariants (checkerboard groups, plaquettes, translations),
  * the free-fermion limit RT = 0,
  * the dense product (I + B_Ltrot ... B_1)^-1,
  * the complex-arithmetic rerun (the reference's own ZGEQP3/ZUNGQR/...):
    imaginary parts stay exactly 0 and the two agree to rounding,
  * the exact mu-derivative identity and finite differences of log det,
  * the committed golden fixture (tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from oracle import z2_oracle as zo

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_ranf_closed_form():
    for seed in (12345, 67890, 1, 2 ** 31 - 1, -5, 987654321):
        r = zo.Ranf(seed)
        s = seed % 2 ** 31
        for n in range(1, 200):
            v = r()
            s = (s * zo.IP_RANF) % 2 ** 31
            assert r.state == s
            assert v == s / 2.0 ** 31
            assert 0.0 <= v < 1.0


def test_ranf_first_values_seed_12345():
    # 32-bit signed emulation of ran_imada.f:62-66, written independently
    iq = 12345
    out = []
    for _ in range(5):
        iq = (iq * 48828125) & 0xFFFFFFFF
        if iq & 0x80000000:
            iq = iq - (1 << 32)
        if iq < 0:
            iq = iq + 2147483647 + 1
        out.append(iq / 2.0 ** 31)
    r = zo.Ranf(12345)
    assert [r() for _ in range(5)] == out


@pytest.mark.parametrize("L", [2, 4, 6, 8, 12])
def test_lattice_tables(L):
    lat = zo.Lattice(L, L)
    N = L * L
    for g in range(4):
        assert lat.groups[g].size == N // 2
        assert lat.group_disjoint[g]
    allb = np.sort(np.concatenate(lat.groups))
    assert np.array_equal(allb, np.arange(2 * N))
    # bond_bonds: each bond and its partners close two plaquettes
    for b in range(2 * N):
        for trip in (lat.bond_bonds[b, 1:4], lat.bond_bonds[b, 4:7]):
            sites = lat.bond_list[np.concatenate(([b], trip))].ravel()
            u, cnt = np.unique(sites, return_counts=True)
            if L > 2:
                assert len(u) == 4 and np.all(cnt == 2)
    # imj is a translation-invariant displacement index
    for i in range(N):
        for j in range(N):
            d = lat.imj[i, j]
            assert lat.imj[lat.L_bonds[i, 1], lat.L_bonds[j, 1]] == d


def test_free_fermion_limit():
    for mu in (0.0, 0.3, -0.7):
        p = zo.Params(RT=0.0, J=0.5, h=0.5, mu=mu, Nlx=4, Nly=4, Ltrot=20, beta=2.0, Nwrap=5)
        c = zo.Z2Chain(p, seed=12345)
        c.pre()
        g = 1.0 / (1.0 + np.exp(p.beta * mu))
        assert np.max(np.abs(c.prop.Gr - g * np.eye(16))) < 1e-13


def test_pre_equals_dense_product():
    p = zo.Params(RT=1.0, J=0.5, h=0.5, mu=0.2, Nlx=4, Nly=4, Ltrot=40, beta=4.0, Nwrap=10)
    c = zo.Z2Chain(p, seed=12345)
    c.pre()
    B = np.eye(16)
    for nt in range(p.Ltrot):
        B = (c.opk.dense_B(c.sigma, nt) * c.opmu.expMU_P) @ B
    G = np.linalg.inv(np.eye(16) + B)
    assert np.max(np.abs(G - c.prop.Gr)) < 1e-12


def test_checkerboard_B_symmetric_and_inverse():
    p = zo.Params(RT=1.0, Nlx=4, Nly=4, Ltrot=10, beta=1.0, Nwrap=5)
    c = zo.Z2Chain(p, seed=3)
    B = c.opk.dense_B(c.sigma, 3, 1)
    Bi = c.opk.dense_B(c.sigma, 3, -1)
    assert np.max(np.abs(B - B.T)) < 1e-15
    assert np.max(np.abs(B @ Bi - np.eye(16))) < 1e-14


def test_complex_rerun_matches_real():
    p = zo.Params(RT=1.0, J=0.5, h=0.5, mu=0.1, Nlx=4, Nly=4, Ltrot=20, beta=2.0, Nwrap=5)
    cr = zo.Z2Chain(p, seed=777)
    cc = zo.Z2Chain(p, seed=777, dtype=np.complex128)
    cr.pre(); cc.pre()
    cr.sweep(); cc.sweep()
    assert np.max(np.abs(np.imag(cc.prop.Gr))) == 0.0
    assert np.max(np.abs(np.real(cc.prop.Gr) - cr.prop.Gr)) < 1e-12
    assert np.array_equal(cr.sigma, cc.sigma)
    for k, v in cr.obs.as_dict().items():
        assert abs(cc.obs.as_dict()[k] - v) < 1e-12 * max(1.0, abs(v))


def test_reject_all_drift_is_rounding():
    p = zo.Params(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=4, Nly=4, Ltrot=40, beta=4.0, Nwrap=10)
    c = zo.Z2Chain(p, seed=12345, rng=zo.ReplayStream(np.full(10 ** 5, 1e300)))
    c.pre()
    c.sweep()
    assert c.prop.Xmaxm < 1e-12


def test_logdet_mu_identity_and_fd():
    L = 4
    rng = np.random.default_rng(7)
    rt = 1.0 + 0.05 * rng.standard_normal(2 * L * L)
    p = zo.Params(RT=rt, J=0.5, h=0.5, mu=0.1, Nlx=L, Nly=L, Ltrot=20, beta=2.0, Nwrap=5)
    lat = zo.Lattice(L, L)
    sig, _, _ = zo.seeded_config(p, lat, 31)
    ld, grad, dmu = zo.logdet_grad_oracle(p, sig)
    h = 1e-5

    def f(rtv, mu):
        q = zo.Params(RT=rtv, J=0.5, h=0.5, mu=mu, Nlx=L, Nly=L, Ltrot=20, beta=2.0, Nwrap=5)
        return zo.logdet_one_sector(q, sig)

    fd_mu = (f(rt, 0.1 + h) - f(rt, 0.1 - h)) / (2 * h)
    assert abs(fd_mu - dmu) < 1e-6
    for b in (0, 5, 17, 31):
        e = np.zeros_like(rt)
        e[b] = h
        fd = (f(rt + e, 0.1) - f(rt - e, 0.1)) / (2 * h)
        assert abs(fd - grad[b]) < 1e-6, b


def test_golden_fixture_reproduced():
    path = os.path.join(GOLDEN, "c1_oracle.npz")
    gold = np.load(path)
    from tests.golden.make_golden import run_c1
    out = run_c1()
    for k in gold.files:
        a, b = out[k], gold[k]
        if a.dtype.kind in "iub":
            assert np.array_equal(a, b), k
        else:
            assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b))), k


def test_read_params_format(tmp_path):
    txt = ("0.5  1.0 0.52 0.3 1\n4 4 80 20\n4 4 80\n4 10 1\n.false. 0\n.false. 200\n"
           ".false. 4\n5\n\n# RT, J, h, mu, Q\n")
    f = tmp_path / "paramC_sets.txt"
    f.write_text(txt)
    p = zo.read_params(str(f))
    assert (p.RT, p.J, p.h, p.mu, p.Q) == (0.5, 1.0, 0.52, 0.3, 1.0)
    assert (p.Nlx, p.Nly, p.Ltrot, p.beta, p.Nwrap) == (4, 4, 80, 20.0, 4)
    assert p.dtau == 0.25 and p.Nst == 20 and p.absolute == 5 and not p.is_tau


def _dense_G(c):
    p = c.p
    B = np.eye(p.Lq)
    for nt in range(p.Ltrot):
        B = (c.opk.dense_B(c.sigma, nt) * c.opmu.expMU_P) @ B
    return np.linalg.inv(np.eye(p.Lq) + B)


def test_nranf_rounding():
    class Fixed:
        def __init__(self, v):
            self.v = v

        def __call__(self):
            return self.v
    c = zo.Z2Chain(zo.Params(RT=1.0, J=0.5, h=0.5, Nlx=2, Nly=2, Ltrot=4, beta=0.4, Nwrap=2))
    for v, N, want in ((0.0, 8, 1), (0.999999, 8, 8), (0.25, 8, 3), (0.3125, 8, 3),
                       (0.375, 8, 4), (0.5, 3, 2)):
        c.rng = Fixed(v)
        assert c.nranf(N) == want, (v, N)


def test_global_moves_keep_G_consistent():
    """Global Wolff-in-tau moves (src/global_update.f90): after each move the
    current G is (I + B_Ltrot ... B_1)^-1 of the current sigma (up to the
    drift of the flips), moves are both accepted and rejected, and the
    direction flag flips on every accepted move."""
    p = zo.Params(RT=1.0, J=0.5, h=0.3, mu=0.1, Nlx=4, Nly=4, Ltrot=20, beta=2.0, Nwrap=5)
    c = zo.Z2Chain(p, seed=4242)
    c.pre()
    seen = set()
    for _ in range(6):
        beta_before = c.is_beta
        c.global_sweep(1)
        acc = c.g_log[-1][4]
        seen.add(acc)
        assert c.is_beta == (beta_before if not acc else not beta_before)
        G = _dense_G(c)
        assert np.max(np.abs(c.prop.Gr - G)) < 1e-6
        c.sweep()
    assert seen == {True, False}
    assert 0.0 <= c.gacc <= 6.0
