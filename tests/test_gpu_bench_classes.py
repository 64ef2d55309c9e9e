"""Whole-bin parity on the configuration the benchmark times.

One chain of each of the 12 (L, beta) classes of the batched workload
(L in {6, 8, 10, 12}, beta in {8, 12, 16} at dtau 0.1, h ~ U[0.2, 1], K = 0.5,
Nwrap 10) plus the single-chain plain configuration (L = 8, beta = 10, 100
slices) run side by side in ONE batched launch, with the delayed-update
ranks and flush tile shapes the library's autotuner picks, exactly as
bench.py builds them.  Each
chain is compared over a whole bin (Local_sweep with Nsweep = 1:
src/local_sweep.f90:152-195; flips src/localK.f90:45-173; stabilization
src/stabilization.f90:122-200, 400-476) with the C restatement of the
reference path (oracle/c/z2cpu.c), started from the same seed:

- accept/reject decisions of both half-sweeps, the links and the ranf state:
  bit-identical;
- G after the bin and the bin's equal-time observables: within 1e-10
  relative (max-abs difference over max-abs value for G; per observable
  against max(|value|, 1));
- the stabilization drift Xmaxm: within 1e-8 relative.  The drift is the
  difference of two nearly equal Green's functions (recomputed minus
  propagated, ~1e-3), so the rounding of each side (~1e-13 of G) is divided
  by a number a thousand times smaller than G.
"""
import numpy as np
import pytest

from bench import batched_chains, single_chain
from oracle import z2cpu
from z2_gauge_zfy_b200 import Z2Batch, tune

pytestmark = pytest.mark.gpu
RTOL = 1e-10
OBS = ("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_shift", "cdw_ratio", "density")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("stab_exact", [False, True], ids=["prepivoted", "pivoted"])
def test_bench_classes_whole_bin_match_c_port(stab_exact):
    """Both stabilizations: the pre-pivoted blocked QR with the scale-split G
    (the default) and the reference's column-pivoted QR (stab_exact)."""
    chains = batched_chains()[:12] + single_chain()
    assert sorted({(c.Nlx, c.Ltrot) for c in chains[:12]}) == \
        [(L, Lt) for L in (6, 8, 10, 12) for Lt in (80, 120, 160)]
    k, shape = tune(chains, stab_exact=stab_exact)
    with Z2Batch(chains, record=True, delay_k_chain=k, flush_shape_chain=shape,
                 stab_exact=stab_exact) as b:
        b.pre()
        b.sweep(1, False)
        gpu = [dict(G=b.green(i), obs=b.obs_equal(i), st=b.stats(i), dec=b.decisions(i)[0],
                    cfg=b.get_config(i)) for i in range(len(chains))]
    worst = {"G": 0.0, "obs": 0.0, "Xmaxm": 0.0}
    for i, ch in enumerate(chains):
        c = z2cpu.CpuChain.from_chain(ch)
        c.pre()
        _, obs, dec = c.bin(record=True)
        st = c.state()
        c.close()
        g = gpu[i]
        tag = f"chain {i} (L={ch.Nlx}, Ltrot={ch.Ltrot}, k={k[i]}, shape={shape[i]})"
        assert np.array_equal(g["dec"], dec), tag
        sig, iseed = g["cfg"]
        assert np.array_equal(sig, st["sigma"]), tag
        assert iseed == st["iseed"], tag
        eg = rel(g["G"], st["G"])
        assert eg < RTOL, (tag, eg)
        for q, name in enumerate(OBS):
            e = abs(g["obs"][name] - obs[q]) / max(abs(obs[q]), 1.0)
            worst["obs"] = max(worst["obs"], e)
            assert e <= RTOL, (tag, name, g["obs"][name], obs[q])
        ex = abs(g["st"]["Xmaxm"] - st["Xmaxm"]) / max(st["Xmaxm"], 1e-12)
        assert ex <= 1e-8, (tag, g["st"]["Xmaxm"], st["Xmaxm"])
        worst["G"] = max(worst["G"], eg)
        worst["Xmaxm"] = max(worst["Xmaxm"], ex)
    print(f"stab_exact={stab_exact}: worst relative differences:", worst)
