"""The allocation-free stab_green entry point, through the C ABI.

Callers whose device memory belongs to another allocator cannot call
cudaMalloc; z2_stab_green_noalloc serves them with a fixed scratch array
inside the library and caller-owned device buffers for inputs and outputs.
This test checks it against the handle-based z2_stab_green and, at the
largest accepted size, against the oracle's stab_green, on the same inputs,
two calls in a row (the scratch keeps the previous call's contents), on both
branches of stab_green, and that sizes beyond the stated maximum are
rejected.  Device buffers for the test's own inputs come from torch.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import z2_oracle as zo
from z2_gauge_zfy_b200 import Chain, Z2Batch, _ffi

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def _inputs(seed):
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=4, Nly=4, Ltrot=40, beta=4.0, Nwrap=10,
               seed=12345)
    p = zo.Params(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=4, Nly=4, Ltrot=40, beta=4.0, Nwrap=10)
    c = zo.Z2Chain(p, seed=ch.seed)
    c.pre()
    st = 2
    UR, DR, VR = c.wr.URlist[st], c.wr.DRlist[st], c.wr.VRlist[st]
    rng = np.random.default_rng(seed)
    UL, _ = np.linalg.qr(rng.standard_normal((p.Lq, p.Lq)))
    DL = np.exp(rng.uniform(-4, 4, p.Lq))
    VL = np.triu(rng.standard_normal((p.Lq, p.Lq))) + 3 * np.eye(p.Lq)
    return ch, (UR, DR, VR, UL, DL, VL)


def _dev(torch, a):
    # column-major device copy
    return torch.tensor(np.ascontiguousarray(np.asarray(a).T), dtype=torch.float64,
                        device="cuda").contiguous()


def test_noalloc_matches_stab_green_twice():
    torch = pytest.importorskip("torch")
    lib = _ffi.load()
    for nt in (10, 30):                      # nt <= Ltrot/2 and nt > Ltrot/2
        ch, mats = _inputs(seed=nt)
        with Z2Batch([ch]) as b:
            ref = b.stab_green(0, *mats, nt)
        N = ch.N
        d = [_dev(torch, m) for m in mats]
        for call in range(2):
            G = torch.full((N, N), float("nan"), dtype=torch.float64, device="cuda")
            rc = lib.z2_stab_green_noalloc(N, nt, ch.Ltrot, *[C.c_void_p(x.data_ptr()) for x in d],
                                           C.c_void_p(G.data_ptr()), None)
            assert rc == 0
            torch.cuda.synchronize()
            got = G.cpu().numpy().T      # column-major back to natural indexing
            err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
            assert err < RTOL, (nt, call, err)


def test_noalloc_rejects_oversize():
    lib = _ffi.load()
    n = _ffi.Z2_NOALLOC_NMAX + 1
    dummy = C.c_void_p(16)       # never dereferenced: the size check comes first
    rc = lib.z2_stab_green_noalloc(n, 1, 10, dummy, dummy, dummy, dummy, dummy, dummy, dummy,
                                   None)
    assert rc == 1               # Z2_ERR_ARG


def _chain_stacks(L, Ltrot, Nwrap, seed):
    """UDV stacks of a real chain: the right chain of Local_sweep_pre and the
    left chain of one left half-sweep (the operands stab_green receives)."""
    p = zo.Params(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=L, Nly=L, Ltrot=Ltrot, beta=0.1 * Ltrot,
                  Nwrap=Nwrap)
    c = zo.Z2Chain(p, seed=seed)
    c.pre()
    wr = c.wr
    right = [(wr.URlist[s].copy(), wr.DRlist[s].copy(), wr.VRlist[s].copy())
             for s in range(p.Nst + 1)]
    c.nobs = 0
    c.sweep_L()
    left = [(wr.ULlist[s].copy(), wr.DLlist[s].copy(), wr.VLlist[s].copy())
            for s in range(p.Nst + 1)]
    return right, left


def test_noalloc_at_max_size():
    """N = 144, the largest size the entry point accepts, on both branches of
    stab_green (nt <= Ltrot/2 and nt > Ltrot/2), on the UDV stacks of a real
    12 x 12 chain: against the oracle's stab_green (a restatement of
    src/stabilization.f90:122-200) and against the handle-based
    z2_stab_green, two calls in a row."""
    torch = pytest.importorskip("torch")
    lib = _ffi.load()
    N = _ffi.Z2_NOALLOC_NMAX
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=12, Nly=12, Ltrot=40, beta=4.0, Nwrap=10,
               seed=4242)
    assert ch.N == N
    right, left = _chain_stacks(12, 40, 10, ch.seed)
    with Z2Batch([ch]) as b:
        for nt in (10, 30):
            st = nt // ch.Nwrap
            mats = (*right[st], *left[st])
            t = zo.Propagator(N)
            t.UUR, t.DUR, t.VUR, t.UUL, t.DUL, t.VUL = mats
            ref_o = zo.stab_green(t, nt, ch.Ltrot)
            ref = b.stab_green(0, *mats, nt)
            d = [_dev(torch, m) for m in mats]
            for call in range(2):
                G = torch.full((N, N), float("nan"), dtype=torch.float64, device="cuda")
                rc = lib.z2_stab_green_noalloc(N, nt, ch.Ltrot,
                                               *[C.c_void_p(x.data_ptr()) for x in d],
                                               C.c_void_p(G.data_ptr()), None)
                assert rc == 0
                torch.cuda.synchronize()
                got = G.cpu().numpy().T
                err_o = np.max(np.abs(got - ref_o)) / np.max(np.abs(ref_o))
                err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
                assert err_o < RTOL, (nt, call, err_o)
                assert err < RTOL, (nt, call, err)
