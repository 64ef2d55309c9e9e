"""Benchmark: spacetime site-updates/s of the DQMC local sweep on B200.

Workload (default): 256 independent Markov chains in one persistent launch,
uneven sizes L in {6, 8, 10, 12} (N = 36..144), beta in {8, 12, 16} at
dtau = 0.1 (Ltrot 80/120/160), h ~ U[0.2, 1.0], K = J = 0.5, t = 1, mu = 0,
seeded +-1 links (conf_set absolute = 1), Nwrap = 10.  A step is one bin
(Local_sweep with Nsweep = 1: sweep_L + sweep_R) of every chain; one
site-update is one (site, slice) visit of a half-sweep, so a chain counts
2 * N * Ltrot site-updates per step.  The single-chain plain path (L = 8,
beta = 10, Ltrot = 100) is measured in the same run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank runs its own 256 chains (seeds offset by rank):
chains are independent, so the path shards with no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DTAU = 0.1
# DRAM bytes (read + write) of one step of the 256-chain workload, from one
# ncu capture of the chain kernel (dram__bytes_read.sum + dram__bytes_write.sum)
TRAFFIC_BYTES_PER_STEP = 2995005440 + 5308945664


def batched_chains(rank: int = 0, n: int = 256):
    from z2_gauge_zfy_b200 import Chain
    rng = np.random.default_rng(20240 + rank)
    hs = rng.uniform(0.2, 1.0, n)
    out = []
    for i in range(n):
        L = (6, 8, 10, 12)[i % 4]
        beta = (8.0, 12.0, 16.0)[(i // 4) % 3]
        out.append(Chain(RT=1.0, J=0.5, h=float(hs[i]), mu=0.0, Nlx=L, Nly=L,
                         Ltrot=int(round(beta / DTAU)), beta=beta, Nwrap=10, absolute=1,
                         seed=12345 + rank * 100003 + i))
    return out


def single_chain():
    from z2_gauge_zfy_b200 import Chain
    return [Chain(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=8, Nly=8, Ltrot=100, beta=10.0, Nwrap=10,
                  absolute=1, seed=12345)]


def adjoint_cost(device: int) -> dict:
    """Cost of the log-det adjoint (z2_logdet_grad) against one sweep of the
    same chain, both timed end to end through the API (median of 3)."""
    from z2_gauge_zfy_b200 import Chain, Z2Batch
    L = 12
    rng = np.random.default_rng(4)
    rt = 1.0 + 0.05 * rng.standard_normal(2 * L * L)
    ch = Chain(RT=1.0, J=0.5, h=0.5, mu=0.1, Nlx=L, Nly=L, Ltrot=120, beta=12.0, Nwrap=10,
               seed=20250, rt_bond=rt)
    with Z2Batch([ch], device=device) as b:
        b.logdet_grad(0)
        tg = []
        for _ in range(3):
            t0 = time.perf_counter()
            b.logdet_grad(0)
            tg.append(time.perf_counter() - t0)
        b.pre()
        b.sweep(1, False)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            b.sweep(1, False)
            ts.append(time.perf_counter() - t0)
    g, s_ = statistics.median(tg), statistics.median(ts)
    return {"workload": "L=12 (N=144), beta=12, dtau 0.1, Ltrot 120, per-bond t = 1 + 0.05 N(0,1), "
                        "mu=0.1, seeded +-1 links, gradient wrt 288 t_b and mu",
            "logdet_grad_ms": g * 1e3, "sweep_ms": s_ * 1e3, "grad_over_sweep": g / s_}


def large_batched(device: int) -> dict:
    """The large batched production configuration: 64 chains, L=16 (N=256),
    beta=20 at dtau 0.05 (400 slices), h=0.6, Nwrap 8, delayed rank 32
    requested, time-displaced G(tau,0) for every tau and the momentum-space
    correlators read back.  One warm-up bin, one timed bin (CUDA events)."""
    from z2_gauge_zfy_b200 import Chain, Z2Batch
    chains = [Chain(RT=1.0, J=0.5, h=0.6, mu=0.0, Nlx=16, Nly=16, Ltrot=400, beta=20.0, Nwrap=8,
                    absolute=1, seed=777 + i) for i in range(64)]
    with Z2Batch(chains, device=device, delay_k=32, tau=True) as b:
        b.pre()
        b.sweep(1, True)
        ms = b.sweep_timed(1, True)
        t0 = time.perf_counter()
        for i in range(len(chains)):
            b.obs_tau_k(i)
        tk = time.perf_counter() - t0
    su = site_updates(chains)
    return {"workload": "64 chains, L=16 (N=256), beta=20, dtau 0.05, Ltrot 400, h=0.6, K=0.5, "
                        "Nwrap 8, delayed rank 32 requested (24 fits shared memory), "
                        "G(tau,0) for all tau + momentum-space correlators",
            "value": su / (ms / 1e3), "unit": "site-updates/s", "ms_per_bin": ms,
            "tau_rate": len(chains) * 256 * 400 / (ms / 1e3), "tau_rate_unit": "(site, tau)/s",
            "momentum_readback_ms": tk * 1e3}


def site_updates(chains) -> int:
    return sum(2 * c.N * c.Ltrot for c in chains)


def algorithmic_flops(chains, acc_rate: float) -> float:
    """FP64 flops of one step (one spin sector), per site-update:
    wrap 72N, updates 8 a N^2, stabilization 14 N^2 / Nwrap, observables 20N."""
    f = 0.0
    for c in chains:
        N = c.N
        per = 72.0 * N + 8.0 * acc_rate * N * N + 14.0 * N * N / c.Nwrap + 20.0 * N
        f += per * 2 * N * c.Ltrot
    return f


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f)
    except OSError:
        return {}


FP64_PEAK_NOTE = ("measured cuBLAS DGEMM 8192^3 (torch.matmul float64) on this pool, "
                  "profiles/fp64_peak_b200.md")


def fp64_peak_tflops():
    """FP64 denominator: measured DGEMM throughput committed under profiles/."""
    path = os.path.join(ROOT, "profiles", "fp64_peak_b200.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["dgemm_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 40.0, "nominal (B200 datasheet FP64 tensor, not measured)"


def _cpu_one(arg):
    """One chain on one core with the C restatement: pre, then one bin timed."""
    c, nbins = arg
    from oracle import z2cpu
    r = z2cpu.run(RT=c.RT, J=c.J, h=c.h, mu=c.mu, beta=c.beta, Nlx=c.Nlx, Nly=c.Nly,
                  Ltrot=c.Ltrot, Nwrap=c.Nwrap, seed=c.seed, nbins=nbins, absolute=c.absolute)
    return 2 * c.N * c.Ltrot * nbins, r["seconds"]


def cpu_baseline_sample():
    """The C restatement of the reference path (reference LAPACK, 1 thread)
    on a stratified sample of the batched workload: one chain of each of the
    12 (L, beta) classes, one bin each."""
    chains = batched_chains()[:12]
    su = sec = 0.0
    for c in chains:
        a, b = _cpu_one((c, 1))
        su += a
        sec += b
    return {"value": su / sec, "unit": "site-updates/s", "cores": 1, "kind": "port",
            "sample": "C restatement (oracle/c/z2cpu.c, reference LAPACK via OpenBLAS, 1 thread, "
                      "one spin sector, real arithmetic: a lower bound on the reference's cost), "
                      "one bin of one chain of each of the 12 (L, beta) classes"}


def run_reference(args):
    """Reference arm: the C restatement of the reference path on all host
    cores, one chain per process (the reference runs one chain per MPI rank)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    from oracle import build_cpu
    build_cpu.build()
    cores = os.cpu_count() or 1
    chains = batched_chains()
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        for w in range(args.warmup):
            pool.map(_cpu_one, [(c, 1) for c in chains[:cores]])
        su_tot = t_tot = 0.0
        for step in range(args.steps):
            # each step: one bin of `cores` chains in parallel; the step's time
            # is the slowest process (all start together)
            sample = [chains[(step * cores + i) % len(chains)] for i in range(cores)]
            res = pool.map(_cpu_one, [(c, 1) for c in sample])
            su_tot += sum(r[0] for r in res)
            t_tot += max(r[1] for r in res)
    v = su_tot / t_tot
    line = {"impl": "reference", "metric": "spacetime site-updates/s", "value": v,
            "unit": "site-updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_tot * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded +-1 links, conf_set absolute=1)",
            "config": {"workload": "batched: chains L in {6,8,10,12}, beta in {8,12,16}, dtau 0.1, "
                                   "h~U[0.2,1], K=0.5, Nwrap 10, one bin per chain; reference arm "
                                   f"runs {cores} chains per step, one per host core"},
            "cpu_baseline": {"value": v, "unit": "site-updates/s", "cores": cores, "kind": "port",
                             "sample": f"{cores} chains x 1 bin per step, one chain per process, "
                                       "C restatement with reference LAPACK (1 BLAS thread each)"},
            "e2e": {"value": v, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--chains", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-single", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    import __graft_entry__
    __graft_entry__.build()
    from z2_gauge_zfy_b200 import Z2Batch, tune_delay

    chains = batched_chains(rank, args.chains)
    su_step = site_updates(chains)
    # delayed-update rank per lattice size from the library's autotuner
    # (short probe chains, before the timed region)
    t_tune = time.perf_counter()
    kchain = tune_delay(chains, local)
    t_tune = time.perf_counter() - t_tune
    b = Z2Batch(chains, device=local, delay_k_chain=kchain)
    b.pre()
    for _ in range(args.warmup):
        b.sweep(1, False)

    def barrier():
        if dist is not None:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    # Timed region: K steps.  Each step is one z2_sweep launch timed with CUDA
    # events on the library's stream (value), and the same step measured end
    # to end through the public API: launch + readback of every chain's bin
    # observables into host memory, wall clock (e2e).  The Markov chains
    # evolve (acceptance falls), so both use the same steps.
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    ms, wall = [], []
    a_num = a_den = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ms.append(b.sweep_timed(1, False))
        for i in range(len(chains)):
            b.obs_equal(i)
        wall.append(time.perf_counter() - t0)
        st = [b.stats(i) for i in range(len(chains))]
        a_num += sum(s["accepted"] for s in st)
        a_den += sum(s["proposed"] for s in st)
    barrier()
    clocks = sampler.stop()
    dev_s = sum(ms) / 1e3
    e2e_s = sum(wall)
    a_rate = a_num / max(a_den, 1.0)

    if dist is not None:
        import torch
        t = torch.tensor([dev_s, e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s, e2e_s = float(t[0]), float(t[1])

    total_su = su_step * args.steps * world
    value = total_su / dev_s
    e2e = total_su / e2e_s
    flops_launch = algorithmic_flops(chains, a_rate)
    launch_s = dev_s / args.steps
    peak, peak_kind = fp64_peak_tflops()
    achieved = flops_launch / launch_s / 1e12
    line = {
        "metric": "spacetime site-updates/s", "value": value, "unit": "site-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded +-1 links, conf_set absolute=1)",
        "config": {"workload": "batched: 256 chains per GPU, L in {6,8,10,12}, beta in "
                               "{8,12,16}, dtau 0.1, h~U[0.2,1], K=J=0.5, t=1, mu=0, Nwrap 10, "
                               "one bin (sweep_L+sweep_R) per step",
                   "chains_per_gpu": len(chains), "site_updates_per_step_per_gpu": su_step,
                   "parallelism": f"chains sharded over {world} GPU(s), replicas",
                   "l2": "inputs larger than L2 (per-GPU chain state > 126 MB)",
                   "accept_rate": a_rate,
                   "delay_rank": {str(c.N): int(k) for c, k in zip(chains, kchain)},
                   "autotune_s": t_tune},
        "e2e": {"value": e2e, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": len(chains) * 7 * 8},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": TRAFFIC_BYTES_PER_STEP if len(chains) == 256 else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                       "bench step (256 chains)",
                     "note": f"FP64 algorithmic flops per launch / launch time; peak {peak_kind}"},
    }
    b.close()
    if rank == 0 and not args.no_single:
        sb = Z2Batch(single_chain(), device=local)
        sb.pre()
        for _ in range(2):
            sb.sweep(1, False)
        sms = [sb.sweep_timed(1, False) for _ in range(3)]
        sv = site_updates(single_chain()) / (sum(sms) / 1e3 / len(sms))
        sb.close()
        line["single_chain"] = {"workload": "L=8 (N=64), beta=10, dtau 0.1, Ltrot 100, h=0.5, "
                                            "K=0.5, one chain", "value": sv,
                                "unit": "site-updates/s",
                                "batched_over_single_per_gpu": (value / world) / sv}
    if rank == 0 and not args.no_single:
        line["adjoint"] = adjoint_cost(local)
        line["large_batched"] = large_batched(local)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
