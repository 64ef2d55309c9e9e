"""The oracle against the reference's own recorded run (test_run/ of the
reference, extracted into tests/golden/testrun_ref.json by
tests/golden/make_testrun_golden.py).

That run is 100 bins of Global_sweep (Nglobal = 4 Wolff moves) followed by
Local_sweep on a 4x4 lattice at beta = 2, Ltrot = 40, Nwrap = 5, mu = 0.3,
absolute = 5, seed 12439 (src/main.f90:72-79).  Replaying it with the same
inputs, the oracle must give the same six per-bin observable series and the
same acceptance figures.  The acceptance ratios are averages of exact
fractions, so they agree only if every local and global accept/reject
decision agrees; the observables agree to rounding.
"""
import json
import os

import numpy as np

from oracle import z2_oracle as zo

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "testrun_ref.json")
OBS_RTOL = 1e-12       # observed: 2.3e-14 (pair_sc_q0)
DRIFT_RTOL = 1e-9      # drift figures are differences of G's: observed 7e-13


def test_oracle_replays_reference_run(tmp_path):
    ref = json.load(open(GOLDEN))
    (tmp_path / "paramC_sets.txt").write_text(ref["params_text"])
    p = zo.read_params(str(tmp_path / "paramC_sets.txt"))
    assert (p.Nlx, p.Nly, p.Ltrot, p.Nwrap, p.Nbin, p.is_global, p.Nglobal, p.absolute) == \
        (4, 4, 40, 5, 100, True, 4, 5)
    assert ref["confin_first"] == 0          # fresh start from seeds.txt
    c = zo.Z2Chain(p, seed=ref["seed"])
    c.pre()
    got = {k: [] for k in ref["series"]}
    progress = {}
    for nbc in range(1, p.Nbin + 1):
        c.global_sweep(p.Nglobal)
        c.sweep()
        d = c.obs.as_dict()
        for k in got:
            got[k].append(d[k])
        if nbc % 20 == 0:
            progress[nbc] = (c.acc / nbc, c.gacc / nbc)
    for k, want in ref["series"].items():
        want = np.array(want)
        have = np.array(got[k])
        err = np.abs(have - want) / np.maximum(np.abs(want), 1e-300)
        assert np.all((err < OBS_RTOL) | (have == want)), (k, err.max(), int(err.argmax()))
    for nbc, acc_l, acc_g in ref["progress"]:
        assert np.isclose(progress[nbc][0], acc_l, rtol=1e-15, atol=0), nbc
        assert np.isclose(progress[nbc][1], acc_g, rtol=1e-15, atol=0), nbc
    s = ref["summary"]
    assert np.isclose(c.gsize / p.Nbin, s["Average size of Wolff cluster"], rtol=1e-15)
    assert np.isclose(c.prop.Xmaxm, s["Max diff Matrix"], rtol=DRIFT_RTOL)
    nmean = 2 * p.Nbin * p.Nst * p.Nsweep    # src/main.f90:110-113, one rank
    assert np.isclose(c.prop.Xmeanm / nmean, s["Mean diff Matrix"], rtol=DRIFT_RTOL)
