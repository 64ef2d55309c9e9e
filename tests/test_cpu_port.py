"""The C restatement (CPU baseline) agrees with the NumPy oracle: identical
decisions and ranf state, G and observables to rounding."""
import numpy as np

from oracle import z2_oracle as zo
from oracle import z2cpu


import pytest


@pytest.mark.parametrize("kw, absolute, seed", [
    (dict(RT=1.0, J=0.5, h=0.5, mu=0.1, beta=2.0, Nlx=4, Nly=4, Ltrot=20, Nwrap=5), 1, 2024),
    (dict(RT=1.0, J=0.5, h=0.0, mu=0.1, beta=2.0, Nlx=4, Nly=4, Ltrot=20, Nwrap=5), 1, 2024),
    # the couplings and start of the reference's recorded run (absolute = 5)
    (dict(RT=0.5, J=1.0, h=0.52, mu=0.3, beta=2.0, Nlx=4, Nly=4, Ltrot=40, Nwrap=5), 5, 12439),
    # a lattice size of the batched workload
    (dict(RT=1.0, J=0.5, h=0.6, mu=0.0, beta=2.0, Nlx=6, Nly=6, Ltrot=20, Nwrap=10), 1, 77),
])
def test_c_port_matches_python_oracle(kw, absolute, seed):
    out = z2cpu.run(**kw, seed=seed, nbins=2, absolute=absolute, record=True)
    p = zo.Params(**kw, absolute=absolute)
    c = zo.Z2Chain(p, seed=seed, record_decisions=True)
    c.pre()
    obs = []
    for _ in range(2):
        c.decisions = []
        c.sweep()
        d = c.obs.as_dict()
        obs.append([d[k] for k in ("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_shift",
                                   "cdw_ratio", "density")])
    nb, L = 2 * p.Lq, p.Ltrot
    dd = np.array(c.decisions, dtype=np.uint8).reshape(2, L, nb)
    d_o = np.stack([dd[0][::-1, ::-1], dd[1]])
    assert np.array_equal(out["decisions"], d_o)
    assert out["iseed"] == c.rng.state
    assert np.max(np.abs(out["G"] - c.prop.Gr)) < 1e-12
    assert np.allclose(out["obs"], np.array(obs), rtol=1e-12, atol=1e-13)


def test_persistent_chain_matches_run_and_oracle_sigma():
    """CpuChain (z2cpu_new / pre / bin / state) gives the same bins as
    z2cpu.run, and its links and ranf state after two bins equal the
    oracle's."""
    kw = dict(RT=1.0, J=0.5, h=0.6, mu=0.1, beta=2.0, Nlx=6, Nly=6, Ltrot=20, Nwrap=10)
    out = z2cpu.run(**kw, seed=91, nbins=2, record=True)
    c = z2cpu.CpuChain(**kw, seed=91)
    c.pre()
    obs = [c.bin(record=True) for _ in range(2)]
    st = c.state()
    c.close()
    assert np.array_equal(obs[-1][2], out["decisions"])
    assert np.array_equal(np.stack([o[1] for o in obs]), out["obs"])
    assert np.array_equal(st["G"], out["G"]) and st["iseed"] == out["iseed"]
    p = zo.Params(**kw)
    o = zo.Z2Chain(p, seed=91)
    o.pre()
    o.sweep()
    o.sweep()
    assert np.array_equal(st["sigma"], o.sigma) and st["iseed"] == o.rng.state
