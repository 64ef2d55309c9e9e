"""Global Wolff-in-tau moves (src/global_update.f90, src/globalK.f90) on the
GPU against the oracle, through the C ABI: after every Global_sweep the
configuration, ranf state, G, the acceptance/cluster counters and the
sweep direction agree exactly (G to 1e-10); the local bins that follow run
in the direction the moves left (is_beta) and make the same decisions."""
import numpy as np
import pytest

from oracle import z2_oracle as zo
from z2_gauge_zfy_b200 import Chain, Z2Batch

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _params(ch):
    return zo.Params(RT=ch.RT, J=ch.J, h=ch.h, mu=ch.mu, Nlx=ch.Nlx, Nly=ch.Nly,
                     Ltrot=ch.Ltrot, beta=ch.beta, Nwrap=ch.Nwrap)


def _oracle_decisions(c, L, nb, left_first):
    d = np.array(c.decisions[-2 * L * nb:], dtype=np.uint8).reshape(2, L, nb)
    iL, iR = (0, 1) if left_first else (1, 0)
    return np.stack([d[iL][::-1, ::-1], d[iR]])


@pytest.mark.parametrize("h,mu", [(0.3, 0.1), (0.8, 0.0)])
def test_global_moves_match_oracle(h, mu):
    ch = Chain(RT=1.0, J=0.5, h=h, mu=mu, Nlx=4, Nly=4, Ltrot=20, beta=2.0, Nwrap=5, seed=4242)
    c = zo.Z2Chain(_params(ch), seed=ch.seed, record_decisions=True)
    c.pre()
    seen = set()
    with Z2Batch([ch], record=True) as b:
        b.pre()
        for _ in range(4):
            c.global_sweep(2)
            b.sweep_global(2)
            gs = b.global_stats(0)
            sig, iseed = b.get_config(0)
            assert np.array_equal(sig, c.sigma)
            assert iseed == c.rng.state
            assert rel(b.green(0), c.prop.Gr) < RTOL
            assert (gs["accepted"], gs["proposed"]) == c.g_last
            assert abs(gs["acc"] - c.gacc) <= 1e-12 and abs(gs["size_cluster"] - c.gsize) <= 1e-12
            assert bool(gs["is_beta"]) == c.is_beta
            seen.update(m[4] for m in c.g_log[-2:])
            left_first = c.is_beta
            c.decisions = []
            c.sweep()
            b.sweep(1, False)
            dec, _ = b.decisions(0)
            assert np.array_equal(dec, _oracle_decisions(c, ch.Ltrot, 2 * ch.N, left_first))
            sig, iseed = b.get_config(0)
            assert np.array_equal(sig, c.sigma) and iseed == c.rng.state
            assert rel(b.green(0), c.prop.Gr) < RTOL
    assert seen == {True, False}


@pytest.mark.parametrize("h", [0.5, 0.0])
def test_boson_warmup_matches_oracle(h):
    """Local_sweep_therm (boson-only warm-up) on the GPU: identical
    configuration, ranf state and accepted fraction after 3 sweeps, then a
    bin from the warmed configuration with identical decisions."""
    ch = Chain(RT=1.0, J=0.5, h=h, mu=0.0, Nlx=4, Nly=4, Ltrot=20, beta=2.0, Nwrap=5, seed=77)
    c = zo.Z2Chain(_params(ch), seed=ch.seed, record_decisions=True)
    accs = [c.therm_sweep() for _ in range(3)]
    with Z2Batch([ch], record=True) as b:
        acc = b.therm(3)
        sig, iseed = b.get_config(0)
        assert np.array_equal(sig, c.sigma)
        assert iseed == c.rng.state
        assert abs(acc[0] - np.mean(accs)) <= 1e-12
        c.pre()
        b.pre()
        c.decisions = []
        c.sweep()
        b.sweep(1, False)
        dec, _ = b.decisions(0)
        assert np.array_equal(dec, _oracle_decisions(c, ch.Ltrot, 2 * ch.N, True))
        assert rel(b.green(0), c.prop.Gr) < RTOL
