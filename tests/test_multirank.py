"""The multi-GPU path on CPU: two gloo ranks run the bench's sharding logic (each rank its own seeded batch,
no data-path collective, barrier + max-over-ranks timing) with the oracle standing in for the device."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import helpers as H


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import bench
    from opendihu_b200 import workloads as WL

    class A:
        impl = "reference"   # gloo backend
    w, r, local, pg = bench.dist_setup(A)
    assert (w, r) == (world, rank)
    batch = WL.batched_hh(clamp_rule="vc", n_fibers=8, min_nodes=20, max_nodes=40, seed=rank, end_time=0.2)
    sub = WL.subset(batch, np.arange(2))
    H.complete(sub)
    st, _, _, n = H.run_oracle(sub, n_threads=1)
    bench.barrier(pg)
    t_max = bench.allmax(pg, float(rank + 1))
    total = bench.allmax(pg, float(sub.n_nodes * n))  # every rank reports its own units
    out[rank] = (t_max, int(batch.n_nodes), float(st[0].sum()))
    pg.destroy_process_group()


def test_two_gloo_ranks_shard_independent_batches():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0][0] == out[1][0] == 2.0          # max over ranks
    assert out[0][1] != out[1][1]                 # each rank has its own seeded batch
    assert np.isfinite(out[0][2]) and np.isfinite(out[1][2])
