"""Extract tests/golden/testrun_ref.json from the reference's own recorded run.

The reference ships one run directory, test_run/, written by its own binary:
the input files (paramC_sets.txt, seeds.txt, confin.txt), info.txt of the
last run and the per-bin observable files, to which every run appends one
line per bin.  info.txt describes that last run (4x4 lattice, t = 0.5, J = 1,
h = 0.52, mu = 0.3, beta = 2, Ltrot = 40, Nwrap = 5, 100 bins, global Wolff
moves with Nglobal = 4, absolute = 5, one MPI rank, fresh start from
seeds.txt); the last Nbin lines of each observable file are therefore its
output.  This script copies those inputs and outputs, as the reference wrote
them, into one small fixture:

  params_text     paramC_sets.txt verbatim
  seed            first line of seeds.txt (rank 0)
  confin_first    first token of confin.txt (0: start from seeds)
  series          {flux_avg, chi_flux, pair_sc_q0, cdw_pi, cdw_ratio,
                   density}: the last Nbin values of each file
  progress        [(bin, Accept_Klocal_shift, Accept_Kglobal)] of info.txt
  summary         Average size of Wolff cluster, Accept_Kglobal,
                  Accept_Klocal_shift, Max diff Matrix, Mean diff Matrix

Run in a checkout that has the reference beside it:

    python -m tests.golden.make_testrun_golden <reference root>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SERIES = ("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_ratio", "density")
SUMMARY = ("Average size of Wolff cluster", "Accept_Kglobal", "Accept_Klocal_shift",
           "Max diff Matrix", "Mean diff Matrix")


def _num(s):
    return float(s.replace("D", "E"))


def extract(root):
    run = os.path.join(root, "test_run")
    read = lambda name: open(os.path.join(run, name), encoding="utf-8").read()
    params_text = read("paramC_sets.txt")
    rows = [ln.split() for ln in params_text.splitlines() if ln.split()]
    nbin = int(rows[3][1])
    info = read("info.txt")
    prog = {}
    for m in re.finditer(r"Progress\s+(\d+)\s*:\s*(Accept_Klocal_shift|Accept_Kglobal):\s*(\S+)",
                         info):
        prog.setdefault(int(m.group(1)), {})[m.group(2)] = _num(m.group(3))
    summary = {}
    for key in SUMMARY:
        m = re.search(r"^\s*" + re.escape(key) + r"\s*:\s*(\S+)\s*$", info, flags=re.M)
        summary[key] = _num(m.group(1))
    return {
        "params_text": params_text,
        "seed": int(read("seeds.txt").split()[0]),
        "confin_first": int(read("confin.txt").split()[0]),
        "series": {k: [_num(x) for x in read(k).split()][-nbin:] for k in SERIES},
        "progress": [[b, v["Accept_Klocal_shift"], v["Accept_Kglobal"]]
                     for b, v in sorted(prog.items())],
        "summary": summary,
    }


if __name__ == "__main__":
    data = extract(sys.argv[1])
    with open(os.path.join(HERE, "testrun_ref.json"), "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", os.path.join(HERE, "testrun_ref.json"))
