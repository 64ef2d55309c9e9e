"""Replica plumbing on CPU: two gloo ranks each run their own oracle chains
(distinct seeds), read the bin observables back through the product's
readback path (Z2Batch.obs_equal_all over a stand-in library that serves the
oracle's values, as bench.py reads its batch) and reduce them and the timing
exactly as the GPU ranks do with NCCL."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _ObsLib:
    """Stand-in library: z2_get_obs_equal_all writes the given rows into the
    caller's buffer, as the CUDA library copies every chain's bin observables."""

    def __init__(self, rows):
        self.rows = rows

    def z2_get_obs_equal_all(self, h, buf):
        for c, row in enumerate(self.rows):
            for q, v in enumerate(row):
                buf[7 * c + q] = v
        return 0


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from oracle import z2_oracle as zo
    from z2_gauge_zfy_b200 import api
    from z2_gauge_zfy_b200.replicas import (bin_observables, chain_seed, max_over_ranks,
                                            reduce_bin_observables)
    p = zo.Params(RT=1.0, J=0.5, h=0.5, mu=0.0, Nlx=4, Nly=4, Ltrot=10, beta=1.0, Nwrap=5)
    rows = []
    for i in range(2):
        c = zo.Z2Chain(p, seed=chain_seed(12345, rank, i))
        c.pre()
        c.sweep()
        d = c.obs.as_dict()
        rows.append([d[k] for k in api.OBS_EQ_NAMES])
    b = api.Z2Batch.__new__(api.Z2Batch)       # no z2_create: nothing on a device
    b.lib, b.h, b.chains = _ObsLib(rows), None, [None, None]
    mean = reduce_bin_observables(bin_observables(b))
    tmax = max_over_ranks(1.0 + rank)
    out[rank] = (np.array(rows), mean, tmax)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction():
    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    rows = np.concatenate([out[r][0] for r in range(world)])
    for r in range(world):
        assert np.allclose(out[r][1], rows.mean(axis=0), rtol=1e-14, atol=0)
        assert out[r][2] == 2.0
    # ranks ran different chains
    assert not np.allclose(out[0][0], out[1][0])
