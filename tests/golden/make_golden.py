"""Generate tests/golden/c1_oracle.npz from the CPU oracle.

The Fortran reference cannot be built in this image (no Fortran compiler,
no MPI), so this fixture records the oracle's own output on the CPU-runnable
configuration (L=4, beta=4, dtau=0.1, Nwrap=10, seed 12345) as a regression
pin: the seeded sigma, the ranf state, G after Local_sweep_pre, and after one
bin the decisions, ratios, G and the equal-time observables.

    python -m tests.golden.make_golden
"""
import os

import numpy as np

from oracle import z2_oracle as zo

HERE = os.path.dirname(os.path.abspath(__file__))
C1 = dict(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=4, Nly=4, Ltrot=40, beta=4.0, Nwrap=10)


def run_c1():
    p = zo.Params(**C1)
    c = zo.Z2Chain(p, seed=12345, record_decisions=True)
    out = {"sigma0": c.sigma.astype(np.int8).copy(), "iseed0": np.array([c.rng.state])}
    c.pre()
    out["G_pre"] = c.prop.Gr.copy()
    c.sweep()
    out["decisions"] = np.array(c.decisions, dtype=np.uint8)
    out["ratios"] = np.array(c.ratios)
    out["G_sweep"] = c.prop.Gr.copy()
    out["sigma1"] = c.sigma.astype(np.int8).copy()
    out["iseed1"] = np.array([c.rng.state])
    out["obs"] = np.array([c.obs.as_dict()[k] for k in
                           ("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_shift",
                            "cdw_ratio", "density")])
    out["Xmaxm"] = np.array([c.prop.Xmaxm])
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(HERE, "c1_oracle.npz"), **run_c1())
    print("wrote", os.path.join(HERE, "c1_oracle.npz"))
