"""Multi-GPU replicas: one process per GPU, each running its own batch of
independent Markov chains.

The reference runs one chain per MPI rank and exchanges nothing during a
sweep (src/main.f90:23-25); per bin it averages the six equal-time
observables over ranks (MPI_REDUCE SUM then /ISIZE, src/fourier_trans.f90:
280-315).  Here a rank holds many chains; the bin average is the mean over all
chains of all ranks, done with one all-reduce of a small vector (NCCL on GPU,
gloo on CPU).  There is no collective inside the data path.
"""
from __future__ import annotations

import numpy as np


def chain_seed(base: int, rank: int, index: int) -> int:
    """Seed of chain `index` on `rank`: distinct over ranks and chains (a
    seeds.txt row per chain, as the reference has one per rank)."""
    return base + rank * 100003 + index


def bin_observables(batch) -> np.ndarray:
    """The bin observables of every chain of a ``Z2Batch`` as an array
    [n_chains, 7] in the order of ``OBS_EQ_NAMES`` (``z2_get_obs_equal_all``,
    the fields Obs_equal_ave writes, src/obser_equal.f90:50-71)."""
    return np.asarray(batch.obs_equal_all(), dtype=np.float64)


def reduce_bin_observables(obs: np.ndarray, group=None, device: str = "cpu") -> np.ndarray:
    """Mean over every chain of every rank.  `obs` is [n_local_chains, n_obs]."""
    import torch
    import torch.distributed as dist
    local = np.asarray(obs, dtype=np.float64)
    t = torch.zeros(local.shape[1] + 1, dtype=torch.float64, device=device)
    t[:-1] = torch.from_numpy(local.sum(axis=0)).to(device)
    t[-1] = float(local.shape[0])
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t = t.cpu().numpy()
    return t[:-1] / t[-1]


def max_over_ranks(value: float, group=None, device: str = "cpu") -> float:
    """The slowest rank's time (the job's time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
