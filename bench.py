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

from dataclasses import dataclass

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DTAU = 0.1
WORKLOAD = ("batched: {n} chains per GPU, L in {{6,8,10,12}}, beta in {{8,12,16}}, dtau 0.1, "
            "h~U[0.2,1], K=J=0.5, t=1, mu=0, Nwrap 10, seeded +-1 links (conf_set absolute=1), "
            "one bin (sweep_L+sweep_R) of every chain per step")


@dataclass
class ChainSpec:
    """One chain's parameters (the hot-path lines of paramC_sets.txt and its
    seed); the fields the library's host binding and the C restatement read."""
    RT: float
    J: float
    h: float
    mu: float
    Nlx: int
    Nly: int
    Ltrot: int
    beta: float
    Nwrap: int
    absolute: int
    seed: int
    Q: float = 1.0
    rt_bond: object = None

    @property
    def N(self):
        return self.Nlx * self.Nly


# DRAM bytes (read + write) of one step of the 256-chain workload, from one
# ncu capture of the chain kernel (dram__bytes_read.sum + dram__bytes_write.sum)
TRAFFIC_BYTES_PER_STEP = 3254171904 + 5548485632


def batched_chains(rank: int = 0, n: int = 256):
    rng = np.random.default_rng(20240 + rank)
    hs = rng.uniform(0.2, 1.0, n)
    out = []
    for i in range(n):
        L = (6, 8, 10, 12)[i % 4]
        beta = (8.0, 12.0, 16.0)[(i // 4) % 3]
        out.append(ChainSpec(RT=1.0, J=0.5, h=float(hs[i]), mu=0.0, Nlx=L, Nly=L,
                             Ltrot=int(round(beta / DTAU)), beta=beta, Nwrap=10, absolute=1,
                             seed=12345 + rank * 100003 + i))
    return out


def single_chain():
    return [ChainSpec(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=8, Nly=8, Ltrot=100, beta=10.0,
                      Nwrap=10, absolute=1, seed=12345)]


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


def fp64_peak_tflops(device: int, n: int = 8192, reps: int = 5):
    """FP64 roofline denominator, measured in this run on this GPU: cuBLAS
    DGEMM n^3 through torch.matmul on float64 (the FP64 tensor pipe), best of
    `reps` timed with CUDA events after two warm-up products."""
    import torch
    dev = torch.device("cuda", device)
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def _cpu_cost(c) -> float:
    """Relative CPU cost of one bin of a chain for the C restatement: wraps
    and observables ~ N^2, accepted-flip updates and stabilizations ~ N^3, per
    slice (acceptance ~0.1 on this workload)."""
    n = float(c.N)
    return c.Ltrot * n * n * (92.0 + 0.8 * n + 14.0 * n / c.Nwrap)


def parity_and_cpu_baseline(device: int, kmap: dict, smap: dict) -> tuple[dict, dict]:
    """The metric's accuracy condition, checked on the benched configuration:
    one chain of each of the 12 (L, beta) classes of the batched workload plus
    the single-chain configuration, one bin each in ONE batched launch with
    the tuned delay ranks and flush shapes, against the C restatement of the reference path
    (oracle/c/z2cpu.c, reference LAPACK, 1 thread) from the same seeds.  The
    C restatement's bin times of the 12 batched classes are the 1-core CPU
    baseline.  Returns (parity, cpu_baseline)."""
    from oracle import z2cpu
    from z2_gauge_zfy_b200 import Z2Batch
    chains = batched_chains()[:12] + single_chain()
    ks = [int(kmap.get(c.N, 0)) for c in chains]
    ss = [int(smap.get(c.N, 0)) for c in chains]
    with Z2Batch(chains, device=device, record=True, delay_k_chain=ks, flush_shape_chain=ss) as b:
        b.pre()
        b.sweep(1, False)
        gpu = [(b.green(i), b.obs_equal(i), b.stats(i)["Xmaxm"], b.decisions(i)[0],
                b.get_config(i)) for i in range(len(chains))]
    g_err = o_err = x_err = 0.0
    dec_same = cfg_same = True
    su = sec = 0.0
    for i, c in enumerate(chains):
        cc = z2cpu.CpuChain.from_chain(c)
        cc.pre()
        t, obs, dec = cc.bin(record=True)
        st = cc.state()
        cc.close()
        G, og, xg, dg, (sig, iseed) = gpu[i]
        g_err = max(g_err, float(np.max(np.abs(G - st["G"])) / np.max(np.abs(st["G"]))))
        ov = np.array(list(og.values()))
        o_err = max(o_err, float(np.max(np.abs(ov - obs) / np.maximum(np.abs(obs), 1.0))))
        x_err = max(x_err, abs(xg - st["Xmaxm"]) / max(st["Xmaxm"], 1e-12))
        dec_same = dec_same and bool(np.array_equal(dg, dec))
        cfg_same = cfg_same and bool(np.array_equal(sig, st["sigma"])) and iseed == st["iseed"]
        if i < 12:
            su += 2 * c.N * c.Ltrot
            sec += t
    parity = {"max_g_rel_err": g_err, "g_err_bound": 1e-8, "g_err_ok": g_err <= 1e-8,
              "decisions_identical": dec_same, "links_and_ranf_identical": cfg_same,
              "max_obs_rel_err": o_err, "max_xmaxm_rel_err": x_err,
              "sample": "one bin of one chain of each of the 12 (L, beta) classes + the "
                        "single-chain configuration (L=8, beta=10), one batched launch with the "
                        "tuned delay ranks, against the C restatement from the same seeds"}
    base = {"value": su / sec, "unit": "site-updates/s", "cores": 1, "kind": "port",
            "sample": "C restatement (oracle/c/z2cpu.c, reference LAPACK via OpenBLAS, 1 thread, "
                      "one spin sector, real arithmetic: a lower bound on the reference's cost), "
                      "one bin of one chain of each of the 12 (L, beta) classes"}
    return parity, base


def _ref_worker(conn, chains):
    """One host core of the reference arm: owns its chains for the whole run
    (the reference keeps a chain in its process between bins), runs Local_sweep
    pre once, then one bin of every owned chain per 'bin' message."""
    from oracle import z2cpu
    cs = [z2cpu.CpuChain.from_chain(c) for c in chains]
    for c in cs:
        c.pre()
    conn.send("ready")
    while conn.recv() == "bin":
        for c in cs:
            c.bin()
        conn.send("done")
    for c in cs:
        c.close()


def run_reference(args):
    """Reference arm: the C restatement of the reference path (the reference
    cannot be built in this image: Fortran + MPI) on every host core, on the
    SAME workload as the GPU arm: the 256 chains of the batched workload, each
    step one bin of every chain, timed by wall clock.  Chains are placed on the
    cores longest-first (greedy by estimated cost) and stay there, as the
    reference runs each chain in its own MPI rank (src/main.f90:23-25)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    from oracle import build_cpu
    build_cpu.build()
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    chains = batched_chains(0, args.chains)
    load = [0.0] * cores
    parts = [[] for _ in range(cores)]
    for c in sorted(chains, key=_cpu_cost, reverse=True):
        w = min(range(cores), key=lambda j: load[j])
        parts[w].append(c)
        load[w] += _cpu_cost(c)
    ctx = mp.get_context("spawn")
    conns, procs = [], []
    for part in parts:
        a, b = ctx.Pipe()
        pr = ctx.Process(target=_ref_worker, args=(b, part), daemon=True)
        pr.start()
        conns.append(a)
        procs.append(pr)
    for a in conns:
        if a.recv() != "ready":
            raise RuntimeError("reference worker failed to start")

    def step():
        t0 = time.perf_counter()
        for a in conns:
            a.send("bin")
        for a in conns:
            if a.recv() != "done":
                raise RuntimeError("reference worker failed")
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    t_tot = sum(step() for _ in range(args.steps))
    for a in conns:
        a.send("stop")
    for pr in procs:
        pr.join(timeout=30)
    su_step = site_updates(chains)
    v = su_step * args.steps / t_tot
    line = {"impl": "reference", "metric": "spacetime site-updates/s", "value": v,
            "unit": "site-updates/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_tot * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded +-1 links, conf_set absolute=1)",
            "config": workload_config(chains),
            "cpu_baseline": {"value": v, "unit": "site-updates/s", "cores": cores, "kind": "port",
                             "sample": f"the whole workload every step: {len(chains)} chains x 1 "
                                       f"bin on {cores} processes (one per host core, chains "
                                       "resident, placed longest-first), wall clock; C "
                                       "restatement with reference LAPACK, 1 BLAS thread each"},
            "e2e": {"value": v, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(chains) -> dict:
    """The `config` of both arms' lines: the workload only."""
    return {"workload": WORKLOAD.format(n=len(chains)), "chains_per_gpu": len(chains),
            "site_updates_per_step_per_gpu": site_updates(chains),
            "l2": "inputs larger than L2 (per-GPU chain state > 126 MB)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--chains", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-single", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="built-in delay ranks and tile shapes (few launches: profiling runs)")
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

    # one build per node: local rank 0 compiles (if the tree is stale), the
    # other ranks wait at a barrier and then load the built library
    if local == 0:
        import __graft_entry__
        __graft_entry__.build()
    if dist is not None:
        dist.barrier()
    from z2_gauge_zfy_b200 import FLUSH_SHAPES, Z2Batch, load, tune
    load()

    chains = batched_chains(rank, args.chains)
    su_step = site_updates(chains)
    # delayed-update rank and flush tile shape per lattice size from the
    # library's autotuner (short probe chains, before the timed region)
    t_tune = time.perf_counter()
    if args.no_tune:
        kchain = np.zeros(len(chains), dtype=np.int32)
        schain = np.zeros(len(chains), dtype=np.int32)
    else:
        kchain, schain = tune(chains, local)
    t_tune = time.perf_counter() - t_tune
    b = Z2Batch(chains, device=local, delay_k_chain=kchain, flush_shape_chain=schain)
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
        b.obs_equal_all()
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

    # bin observables of every chain of every rank, averaged as the reference
    # averages them over its MPI ranks (one all-reduce after the timed region)
    from z2_gauge_zfy_b200.replicas import bin_observables, reduce_bin_observables
    obs_local = bin_observables(b)
    obs_mean = reduce_bin_observables(obs_local, device=f"cuda:{local}" if dist else "cpu")

    total_su = su_step * args.steps * world
    value = total_su / dev_s
    e2e = total_su / e2e_s
    flops_launch = algorithmic_flops(chains, a_rate)
    launch_s = dev_s / args.steps
    b.close()
    peak = fp64_peak_tflops(local)
    achieved = flops_launch / launch_s / 1e12
    kmap = {c.N: int(k) for c, k in zip(chains, kchain)}
    smap = {c.N: int(x) for c, x in zip(chains, schain)}
    line = {
        "metric": "spacetime site-updates/s", "value": value, "unit": "site-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded +-1 links, conf_set absolute=1)",
        "config": workload_config(chains),
        "parallelism": f"chains sharded over {world} GPU(s), replicas",
        "accept_rate": a_rate,
        "delay_rank": ",".join(f"N{n}:k{k}" for n, k in sorted(kmap.items())),
        "flush_shape": ",".join(f"N{n}:{FLUSH_SHAPES[x]}" for n, x in sorted(smap.items())),
        "tuning": "z2_tune: ranks 4..64 (shared memory caps them: k <= 8 at N = 144) x every "
                  "flush tile shape valid for N, median SM cycles of 3 probe chains, first "
                  "within 3 % of the fastest in the order (default shape, smaller rank)",
        "autotune_s": t_tune,
        "bin_observables_mean": dict(zip(("flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi",
                                          "cdw_shift", "cdw_ratio", "density"),
                                         obs_mean.tolist())),
        "e2e": {"value": e2e, "unit": "site-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": len(chains) * 7 * 8},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": TRAFFIC_BYTES_PER_STEP if len(chains) == 256 else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                       "bench step (256 chains)",
                     "note": "FP64 algorithmic flops per launch / launch time; peak = cuBLAS "
                             "DGEMM 8192^3 (torch.matmul float64) measured in this run"},
    }
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
    if rank == 0:
        parity, base = parity_and_cpu_baseline(local, kmap, smap)
        line["parity"] = parity
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = base
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
