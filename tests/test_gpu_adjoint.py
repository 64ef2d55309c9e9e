"""Adjoint of log det(1 + B_Ltrot ... B_1) on the B200 path at the full
adjoint configuration (L = 12, beta = 12, dtau 0.1, 120 slices, per-bond
hopping 1 + 0.05 N(0,1), mu = 0.1, seeded +-1 links, UDV checkpoints every
10 slices), checked against central finite differences of the library's own
log det (step 1e-5).  The reference has no adjoint; its log det is the
quantity whose derivative is taken (src/stabilization.f90 stab_green chain).
"""
import numpy as np
import pytest

from z2_gauge_zfy_b200 import Chain, Z2Batch

pytestmark = pytest.mark.gpu

L, BETA, LT, NWRAP, MU = 12, 12.0, 120, 10, 0.1
FD_STEP = 1e-5
FD_TOL = 1e-6


def _chain(rt, mu=MU):
    return Chain(RT=1.0, J=0.5, h=0.5, mu=mu, Nlx=L, Nly=L, Ltrot=LT, beta=BETA, Nwrap=NWRAP,
                 seed=20250, rt_bond=rt)


def _logdet(rt, mu=MU):
    with Z2Batch([_chain(rt, mu)]) as b:
        return b.logdet_grad(0)


def test_adjoint_matches_central_differences():
    N = L * L
    rng = np.random.default_rng(4)
    rt = 1.0 + 0.05 * rng.standard_normal(2 * N)
    ld, g, dmu = _logdet(rt)
    assert g.shape == (2 * N,) and np.all(np.isfinite(g))
    bonds = rng.choice(2 * N, size=8, replace=False)
    for bnd in bonds:
        rp, rm = rt.copy(), rt.copy()
        rp[bnd] += FD_STEP
        rm[bnd] -= FD_STEP
        fd = (_logdet(rp)[0] - _logdet(rm)[0]) / (2 * FD_STEP)
        assert abs(g[bnd] - fd) <= FD_TOL * max(1.0, abs(fd)), (bnd, g[bnd], fd)
    fd_mu = (_logdet(rt, MU + FD_STEP)[0] - _logdet(rt, MU - FD_STEP)[0]) / (2 * FD_STEP)
    assert abs(dmu - fd_mu) <= FD_TOL * max(1.0, abs(fd_mu)), (dmu, fd_mu)
