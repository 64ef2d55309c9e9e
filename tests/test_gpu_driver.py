"""The C++ host driver (restatement of src/main.f90 over the C ABI) on the
reference's own input files, checked against the oracle: per-bin observable
files averaged over chains, confout.txt, and a restart from confin.txt."""
import os
import subprocess

import numpy as np
import pytest

from oracle import z2_oracle as zo
from z2_gauge_zfy_b200 import build

pytestmark = pytest.mark.gpu

PARAMS = ("1.0 0.5 0.5 0.1 1\n4 4 20 2.0\n4 4 20\n10 2 1\n.false. 0\n.false. 0\n"
          ".false. 0\n1\n")


def _run(tmp, nch, confin="0\n", seeds=(12345, 67890)):
    build.build()
    (tmp / "paramC_sets.txt").write_text(PARAMS)
    (tmp / "confin.txt").write_text(confin)
    (tmp / "seeds.txt").write_text("".join(f"{s}\n" for s in seeds))
    r = subprocess.run([build.DRIVER, "--chains", str(nch), "--dir", str(tmp)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    read = lambda n: np.array([float(x) for x in (tmp / n).read_text().split()])
    return {n: read(n) for n in ("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_ratio",
                                 "density")}


def _oracle_bins(p, chains):
    out = {k: [] for k in ("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_ratio", "density")}
    for _ in range(p.Nbin):
        vals = []
        for c in chains:
            c.sweep()
            vals.append(c.obs.as_dict())
        for k in out:
            out[k].append(np.mean([v[k] for v in vals]))
    return {k: np.array(v) for k, v in out.items()}


def test_driver_two_chains_matches_oracle(tmp_path):
    got = _run(tmp_path, 2)
    p = zo.read_params(str(tmp_path / "paramC_sets.txt"))
    chains = [zo.Z2Chain(p, seed=s) for s in (12345, 67890)]
    for c in chains:
        c.pre()
    ref = _oracle_bins(p, chains)
    for k in ref:
        assert np.allclose(got[k], ref[k], rtol=1e-10, atol=1e-12), k
    # confout.txt: iseed then sigma(2N, Ltrot) per chain
    tok = (tmp_path / "confout.txt").read_text().split()
    nb, lt = 2 * p.Lq, p.Ltrot
    per = 1 + nb * lt + p.Lq
    for i, c in enumerate(chains):
        blk = tok[i * per:(i + 1) * per]
        assert int(blk[0]) == c.rng.state
        sig = np.array([float(x) for x in blk[1:1 + nb * lt]]).reshape(lt, nb).T
        assert np.array_equal(sig, c.sigma)


def test_driver_restart_from_confin(tmp_path):
    first = tmp_path / "a"
    first.mkdir()
    _run(first, 1)
    restart = tmp_path / "b"
    restart.mkdir()
    conf = (first / "confout.txt").read_text()
    got = _run(restart, 1, confin=conf)
    p = zo.read_params(str(restart / "paramC_sets.txt"))
    tok = conf.split()
    nb, lt = 2 * p.Lq, p.Ltrot
    sig = np.array([float(x) for x in tok[1:1 + nb * lt]]).reshape(lt, nb).T
    c = zo.Z2Chain(p, sigma=sig, rng=zo.Ranf(int(tok[0])))
    c.pre()
    ref = _oracle_bins(p, [c])
    for k in ref:
        assert np.allclose(got[k], ref[k], rtol=1e-10, atol=1e-12), k


def test_driver_tau_momentum_files(tmp_path):
    """is_tau: the per-bin momentum-space files of m_write_obs_tau
    (src/fourier_trans.f90:306-440), DFT on the GPU, against the oracle."""
    build.build()
    params = PARAMS.replace(".false. 0\n.false. 0\n.false. 0\n", ".true. 0\n.false. 0\n.false. 0\n")
    (tmp_path / "paramC_sets.txt").write_text(params)
    (tmp_path / "confin.txt").write_text("0\n")
    (tmp_path / "seeds.txt").write_text("12345\n")
    r = subprocess.run([build.DRIVER, "--chains", "1", "--dir", str(tmp_path)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    p = zo.read_params(str(tmp_path / "paramC_sets.txt"))
    assert p.is_tau
    c = zo.Z2Chain(p, seed=12345)
    c.pre()
    lat = zo.Lattice(p.Nlx, p.Nly)
    dtau = p.beta / p.Ltrot
    want = {"sdw_zero_susc": [], "cdw_s_pipi_susc": [], "pair_d_zero_susc": [], "g_zero_susc": []}
    src = {"sdw_zero_susc": ("spin", 0), "cdw_s_pipi_susc": ("charge_s", (p.Nly // 2) * p.Nlx + p.Nlx // 2),
           "pair_d_zero_susc": ("pair_d", 0), "g_zero_susc": ("single", 0)}
    for _ in range(p.Nbin):
        c.sweep(toggle=True)
        for f, (name, k) in src.items():
            g = zo.integrate_susc(zo.fourier_r_to_k(c.obs_tau.arr[name], lat), dtau)
            want[f].append(g[k])
    for f, vals in want.items():
        got = np.array([float(x) for x in (tmp_path / f).read_text().split()]).reshape(-1, 2)
        ref = np.array([[v.real, v.imag] for v in vals])
        assert np.allclose(got, ref, rtol=1e-9, atol=1e-12), f
    for f in ("sdw_susc", "curxx_freq", "curxx_L_tau", "g_r0_tau", "pair_s_zero_tau"):
        assert (tmp_path / f).stat().st_size > 0, f


def test_driver_global_moves(tmp_path):
    """is_global: Nglobal Wolff moves before every bin (src/main.f90:76),
    per-bin observables against the oracle doing the same."""
    build.build()
    params = PARAMS.replace(".false. 0\n.false. 0\n.false. 0\n", ".false. 0\n.false. 0\n.true. 2\n")
    (tmp_path / "paramC_sets.txt").write_text(params)
    (tmp_path / "confin.txt").write_text("0\n")
    (tmp_path / "seeds.txt").write_text("12345\n")
    r = subprocess.run([build.DRIVER, "--chains", "1", "--dir", str(tmp_path)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    p = zo.read_params(str(tmp_path / "paramC_sets.txt"))
    assert p.is_global and p.Nglobal == 2
    c = zo.Z2Chain(p, seed=12345)
    c.pre()
    ref = {k: [] for k in ("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_ratio", "density")}
    for _ in range(p.Nbin):
        c.global_sweep(p.Nglobal)
        c.sweep()
        d = c.obs.as_dict()
        for k in ref:
            ref[k].append(d[k])
    for k, v in ref.items():
        got = np.array([float(x) for x in (tmp_path / k).read_text().split()])
        assert np.allclose(got, np.array(v), rtol=1e-10, atol=1e-12), k
    info = (tmp_path / "info.txt").read_text()
    assert "Accept_Kglobal" in info and "Wolff cluster" in info


def test_driver_warm_up(tmp_path):
    """is_warm: Nwarm boson-only sweeps (Local_sweep_therm, src/main.f90:38-67)
    on the GPU before Local_sweep_pre, then per-bin observables against the
    oracle doing the same."""
    build.build()
    params = PARAMS.replace(".false. 0\n.false. 0\n.false. 0\n", ".false. 0\n.true. 3\n.false. 0\n")
    (tmp_path / "paramC_sets.txt").write_text(params)
    (tmp_path / "confin.txt").write_text("0\n")
    (tmp_path / "seeds.txt").write_text("12345\n")
    r = subprocess.run([build.DRIVER, "--chains", "1", "--dir", str(tmp_path)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    p = zo.read_params(str(tmp_path / "paramC_sets.txt"))
    assert p.is_warm and p.Nwarm == 3
    c = zo.Z2Chain(p, seed=12345)
    for _ in range(p.Nwarm):
        c.therm_sweep()
    c.pre()
    ref = _oracle_bins(p, [c])
    for k in ref:
        got = np.array([float(x) for x in (tmp_path / k).read_text().split()])
        assert np.allclose(got, ref[k], rtol=1e-10, atol=1e-12), k
