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


class LogDet:
    """log|det(1 + B_Ltrot ... B_1)| of one spin sector as a function of the
    per-bond hoppings and mu, with the library's hand-written adjoint
    (z2_logdet_grad, through the C ABI) as its backward.  Test harness only:
    the product is the C ABI."""

    @staticmethod
    def function():
        import torch

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, t, mu):
                ld, g, dmu = _logdet(t.detach().cpu().numpy().astype(np.float64),
                                     float(mu.detach().cpu()))
                ctx.save_for_backward(torch.from_numpy(g).to(t), torch.tensor(dmu).to(mu))
                return torch.tensor(ld, dtype=torch.float64)

            @staticmethod
            def backward(ctx, gout):
                g, dmu = ctx.saved_tensors
                return gout * g, gout * dmu

        return _F.apply


def test_autograd_wrapper_backpropagates_the_adjoint():
    """A loss built on the log det backpropagates through the adjoint kernel:
    loss = log det / 2 + sum(t^2) + mu^2, whose gradient is checked by central
    finite differences of the same loss (step 1e-5) on eight bonds and mu."""
    torch = pytest.importorskip("torch")
    logdet = LogDet.function()
    N = L * L
    rng = np.random.default_rng(4)
    rt = 1.0 + 0.05 * rng.standard_normal(2 * N)

    def loss_np(r, m):
        return 0.5 * _logdet(r, m)[0] + float(np.sum(r * r)) + m * m

    t = torch.tensor(rt, dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(MU, dtype=torch.float64, requires_grad=True)
    loss = 0.5 * logdet(t, mu) + (t * t).sum() + mu * mu
    loss.backward()
    gt, gmu = t.grad.numpy(), float(mu.grad)
    for bnd in rng.choice(2 * N, size=8, replace=False):
        rp, rm = rt.copy(), rt.copy()
        rp[bnd] += FD_STEP
        rm[bnd] -= FD_STEP
        fd = (loss_np(rp, MU) - loss_np(rm, MU)) / (2 * FD_STEP)
        assert abs(gt[bnd] - fd) <= FD_TOL * max(1.0, abs(fd)), (bnd, gt[bnd], fd)
    fd_mu = (loss_np(rt, MU + FD_STEP) - loss_np(rt, MU - FD_STEP)) / (2 * FD_STEP)
    assert abs(gmu - fd_mu) <= FD_TOL * max(1.0, abs(fd_mu)), (gmu, fd_mu)
