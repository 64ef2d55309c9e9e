"""Input errors of the C++ host driver (the restatement of src/main.f90),
which the reference meets with a message and `stop`: each one ends the driver
with status 1 and a message before its first library call, so these run
without a GPU."""
import subprocess

import pytest

from z2_gauge_zfy_b200 import build

# paramC_sets.txt: RT J h mu Q / Nlx Nly Ltrot beta / NlxT NlyT LtrotT /
# Nwrap Nbin Nsweep / is_tau Nthermal / is_warm Nwarm / is_global Nglobal / absolute
LINES = ["1.0 0.5 0.5 0.1 1", "4 4 20 2.0", "4 4 20", "10 2 1", ".false. 0", ".false. 0",
         ".false. 0", "1"]


def _params(edit=None):
    """LINES with {(row, field): value} replaced."""
    lines = list(LINES)
    for (row, col), v in (edit or {}).items():
        tok = lines[row].split()
        tok[col] = v
        lines[row] = " ".join(tok)
    return "\n".join(lines) + "\n"


def _run(tmp, params, chains=1, seeds="12345\n", confin="0\n"):
    drv = build.build_driver()
    if params is not None:
        (tmp / "paramC_sets.txt").write_text(params)
    (tmp / "seeds.txt").write_text(seeds)
    (tmp / "confin.txt").write_text(confin)
    r = subprocess.run([drv, "--chains", str(chains), "--dir", str(tmp)], capture_output=True,
                       text=True, timeout=60)
    return r.returncode, r.stderr


@pytest.mark.parametrize("case, kw, msg", [
    ("no parameter file", dict(params=None), "cannot read"),
    ("short line", dict(params="\n".join(LINES[:1] + ["4 4"] + LINES[2:]) + "\n"), "cannot read"),
    ("Nwrap = 0", dict(params=_params({(3, 0): "0"})), "must be >= 1"),
    ("NlxT = 0", dict(params=_params({(2, 0): "0"})), "must be >= 1"),
    ("Nsweep = 0", dict(params=_params({(3, 2): "0"})), "must be >= 1"),
    ("Ltrot not a multiple of Nwrap", dict(params=_params({(1, 2): "25"})), "multiple of Nwrap"),
    ("no chains", dict(params=_params(), chains=0), "--chains"),
    ("too few seeds", dict(params=_params(), chains=2), "fewer than 2 seeds"),
    ("truncated confin", dict(params=_params(), confin="12345\n1.0 -1.0\n"), "truncated"),
])
def test_driver_rejects(tmp_path, case, kw, msg):
    rc, err = _run(tmp_path, **kw)
    assert rc == 1, (case, rc, err)
    assert msg in err, (case, err)


def test_driver_rejects_unwritable_output(tmp_path):
    """An output file that cannot be opened ends the run before any work
    (here info.txt is a directory, which no user can open for writing)."""
    (tmp_path / "info.txt").mkdir()
    rc, err = _run(tmp_path, _params())
    assert rc == 1 and "cannot write" in err, err
