"""Fiber sharding on CPU: the LPT partition, shard subsets, the host-only clamp selection of the library
against the oracle's, shard-local clamp mapping, shard runs of the oracle against the unsharded run, and the
end-of-interval gather over two gloo ranks."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import helpers as H
from opendihu_b200 import _native as N
from opendihu_b200 import sharding as SH
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(3)
    w = rng.integers(500, 2501, size=4096)
    for n in (1, 2, 3, 8):
        parts = SH.lpt_partition(w, n)
        allf = np.sort(np.concatenate(parts))
        np.testing.assert_array_equal(allf, np.arange(len(w)))
        loads = np.array([w[p].sum() for p in parts])
        lower = max(w.sum() / n, w.max())
        assert loads.max() <= 4 / 3 * lower            # Graham's bound for LPT
        assert loads.max() - loads.min() <= w.max()    # no shard above another by more than one fiber
        for p in parts:
            assert np.all(np.diff(p) > 0)
    assert [list(p) for p in SH.lpt_partition([5, 5, 5], 2)] == [[0, 2], [1]]  # ties by index, then shard
    assert [len(p) for p in SH.lpt_partition([1, 2], 4)] == [1, 1, 0, 0]
    with pytest.raises(ValueError):
        SH.lpt_partition([1], 0)


def test_subset_keeps_per_fiber_inputs():
    s = WL.batched_hh(clamp_rule="vc", n_fibers=9, min_nodes=10, max_nodes=30, seed=2, end_time=0.1)
    H.complete(s)
    s.jitter = np.arange(9 * 2, dtype=float).reshape(9, 2)
    fib = np.array([7, 1, 4])
    sub = SH.subset(s, fib)
    off = s.fiber_offsets
    for k, f in enumerate(fib):
        a, b = sub.fiber_offsets[k], sub.fiber_offsets[k + 1]
        np.testing.assert_array_equal(sub.states[:, a:b], s.states[:, off[f]:off[f + 1]])
        np.testing.assert_array_equal(sub.parameters[:, a:b], s.parameters[:, off[f]:off[f + 1]])
        np.testing.assert_array_equal(sub.element_lengths[a - k:b - k - 1], s.element_lengths[off[f] - f:off[f + 1] - f - 1])
        assert sub.motor_unit_no[k] == s.motor_unit_no[f] and sub.prefactor[k] == s.prefactor[f]
        np.testing.assert_array_equal(sub.jitter[k], s.jitter[f])
    np.testing.assert_array_equal(SH.node_index(off, fib),
                                  np.concatenate([np.arange(off[f], off[f + 1]) for f in fib]))


@pytest.mark.parametrize("n_ranks,width", [(1, 4), (2, 4), (3, 8), (1, 2), (4, 1)])
def test_library_clamp_selection_matches_oracle(n_ranks, width):
    s = WL.batched_hh(clamp_rule="vc", n_fibers=23, min_nodes=7, max_nodes=90, seed=n_ranks * 10 + width, end_time=0.0)
    s.n_ranks, s.vc_width = n_ranks, width
    rng = np.random.default_rng(width)
    lengths = np.diff(s.fiber_offsets)
    s.stimulation_point_index = rng.integers(0, lengths).astype(np.int32)
    H.complete(s)
    first, cnt, ev = SH.global_clamp_nodes(s)
    of, oc = H.O.OracleRun(H.oracle_spec(s)).vc_clamp_nodes()
    np.testing.assert_array_equal(first, of)
    np.testing.assert_array_equal(cnt, oc)
    np.testing.assert_array_equal(ev, (of >= 0).astype(np.uint8))


def test_center_rule_selection_and_bad_arguments():
    off = np.array([0, 5, 6, 16], np.int64)
    first, cnt, ev = N.select_clamp_nodes(S.CLAMP_RULES["center"], 4, 1, off, np.array([0, 0, 9], np.int32))
    np.testing.assert_array_equal(first, [0, 5, 14])
    np.testing.assert_array_equal(cnt, [2, 1, 2])
    np.testing.assert_array_equal(ev, [1, 1, 1])
    with pytest.raises(N.FdmError):
        N.select_clamp_nodes(7, 4, 1, off, np.zeros(3, np.int32))
    with pytest.raises(N.FdmError):
        N.select_clamp_nodes(0, 0, 1, off, np.zeros(3, np.int32))


def test_shard_clamp_mapping():
    s = WL.batched_hh(clamp_rule="vc", n_fibers=11, min_nodes=20, max_nodes=60, seed=5, end_time=0.0)
    clamp = SH.global_clamp_nodes(s)
    for fib in SH.lpt_partition(np.diff(s.fiber_offsets), 3):
        lf, lc, le = SH.shard_clamp_nodes(s, fib, clamp)
        sub = SH.subset(s, fib)
        g = SH.node_index(s.fiber_offsets, fib)
        for k, f in enumerate(fib):
            assert lc[k] == clamp[1][f] and le[k] == clamp[2][f]
            if clamp[0][f] >= 0:
                assert g[lf[k]] == clamp[0][f]                                   # same global node
                assert sub.fiber_offsets[k] <= lf[k] < sub.fiber_offsets[k + 1]   # inside the shard's fiber


def test_oracle_shards_equal_unsharded_run():
    # with the layout-independent "center" clamp rule every fiber evolves alone: shard runs of the oracle
    # reproduce the unsharded run bit for bit, the property the sharded solver relies on
    s = WL.batched_hh(n_fibers=7, min_nodes=15, max_nodes=40, seed=4, end_time=0.3, clamp_rule="center")
    H.complete(s)
    full, _, _, n = H.run_oracle(s.copy(), n_threads=1)
    got = np.zeros_like(full)
    for fib in SH.lpt_partition(np.diff(s.fiber_offsets), 3):
        st, _, _, m = H.run_oracle(SH.subset(s, fib), n_threads=1)
        assert m == n
        got[:, SH.node_index(s.fiber_offsets, fib)] = st
    np.testing.assert_array_equal(got, full)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _gather_worker(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = WL.batched_hh(n_fibers=6, min_nodes=12, max_nodes=30, seed=9, end_time=0.2, clamp_rule="center")
        H.complete(s)
        fib, sub, clamp = SH.rank_shard(s, rank, world)
        st, _, _, _ = H.run_oracle(sub, n_threads=1)
        g = SH.gather_to_root(None, s, fib, st[:1])
        if rank == 0:
            out["vm"] = g[0]
        out[rank] = list(map(int, fib))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_shards():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_gather_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    s = WL.batched_hh(n_fibers=6, min_nodes=12, max_nodes=30, seed=9, end_time=0.2, clamp_rule="center")
    H.complete(s)
    full, _, _, _ = H.run_oracle(s.copy(), n_threads=1)
    assert sorted(out[0] + out[1]) == list(range(6))
    np.testing.assert_array_equal(out["vm"], full[0])


def test_shard_gate_codes_map_fibers():
    s = WL.batched_hh(n_fibers=9, min_nodes=20, max_nodes=40, seed=6, end_time=0.0, clamp_rule="center")
    codes = SH.global_gate_codes(s)
    for fib in SH.lpt_partition(np.diff(s.fiber_offsets), 3):
        c = SH.shard_gate_codes(s, fib, codes)
        sub = SH.subset(s, fib)
        want = N.select_gate_codes(S.CLAMP_RULES["center"], 4, 1, sub.fiber_offsets, sub.stimulation_point_index)
        np.testing.assert_array_equal(c, want)
    # vc rule, uneven lengths: some buffer is attributed across a shard boundary
    s.clamp_rule = "vc"
    codes = SH.global_gate_codes(s)
    if np.any((codes >> 2) != np.repeat(np.arange(9), np.diff(s.fiber_offsets))):
        with pytest.raises(ValueError):
            for fib in SH.lpt_partition(np.diff(s.fiber_offsets), 3):
                SH.shard_gate_codes(s, fib, codes)


def test_adjoint_memory_plan():
    s = WL.batched_hh(clamp_rule="vc", n_fibers=40, min_nodes=500, max_nodes=2500, seed=3, end_time=0.0)
    one = SH.adjoint_bytes_per_node(s.model, 5, 1000, 16)
    # checkpoints fall and replay grows with the interval
    assert SH.adjoint_bytes_per_node(s.model, 5, 1000, 1) > one < SH.adjoint_bytes_per_node(s.model, 5, 1000, 500)
    big = SH.plan_adjoint(s, 0.0, 1.0, 1e12)
    assert big["n_shards"] == 1 and big["n_steps"] == 1000
    assert 5 <= big["checkpoint_every"] <= 12           # ~ sqrt(1000 / (4 * 5))
    budget = s.n_nodes * big["bytes_per_node"] / 3.5
    plan = SH.plan_adjoint(s, 0.0, 1.0, budget)
    assert plan["n_shards"] >= 4 and plan["largest_shard_nodes"] * plan["bytes_per_node"] <= budget
    with pytest.raises(ValueError):
        SH.plan_adjoint(s, 0.0, 1.0, 1000.0)
