"""Accuracy of the reduced-precision and fused solvers against the FP64 solvers, on full-size workloads.

The north-star criterion for the FP32-reaction path is a transmembrane-potential error of at most 0.1 mV and
activation times within one split step of the FP64 plain method.  These helpers measure both on the device:
Vm of every node is compared after every chunk of the span, and activation steps (the Strang steps after which
Vm rises above a threshold, recorded by the library on traced nodes: fdm_set_activation_recording) are compared
per traced node.
"""
from __future__ import annotations

import numpy as np

from . import sharding as SH
from . import solver as S


def traced_nodes(system, per_fiber: int) -> np.ndarray:
    """per_fiber nodes of every fiber, evenly spaced from its first to its last node (global node numbers)."""
    off = np.asarray(system.fiber_offsets, np.int64)
    out = [off[f] + np.linspace(0, int(off[f + 1] - off[f]) - 1, per_fiber).round().astype(np.int64)
           for f in range(system.n_fibers)]
    return np.concatenate(out) if out else np.zeros(0, np.int64)


def compare_activation(ca, sa, cb, sb) -> dict:
    """Activation steps of two runs at the same traced nodes (counts [node], steps [node, capacity]): the nodes
    whose numbers of crossings differ, and the largest step difference between the matched crossings of the
    other nodes."""
    ca, cb = np.asarray(ca), np.asarray(cb)
    sa, sb = np.asarray(sa, np.int64), np.asarray(sb, np.int64)
    cap = sa.shape[1]
    same = (ca == cb) & (ca <= cap)
    valid = (np.arange(cap)[None, :] < np.minimum(ca, cap)[:, None]) & same[:, None]
    d = np.abs(sa - sb)
    return {"traced_nodes": int(len(ca)), "crossings": int(cb.sum()), "nodes_with_crossings": int((cb > 0).sum()),
            "nodes_count_mismatch": int((~same).sum()), "max_step_diff": int(d[valid].max()) if valid.any() else 0}


def batch_accuracy(system, device: int = 0, span_ms: float = 100.0, chunk_ms: float = 1.0, per_fiber: int = 32,
                   subset_fibers: int = 64, threshold: float = 0.0) -> dict:
    """The FP32-reaction fused solver against the FP64 fused solver on every fiber of ``system`` over
    [0, span_ms] (Vm of all nodes compared after every chunk_ms; activation steps at per_fiber traced nodes per
    fiber), and the FP64 split solver -- the reference's plain method -- on subset_fibers fibers of the system
    (keeping the clamp nodes of the whole layout, so its fibers are the same problems) against the FP64 fused
    solver's values of those fibers.  Both fused solvers use autotuned launch shapes."""
    from . import workloads as WL
    sysm = system.copy()
    sysm.start_time, sysm.end_time = 0.0, float(span_ms)
    nodes = traced_nodes(sysm, per_fiber)
    runs = {}
    for name, prec in (("fp32_fused", "fp32"), ("fp64_fused", "fp64")):
        runs[name] = S.FastMonodomainSolver(sysm.copy(), method="fused", precision=prec, device=device,
                                            autotune=True, trace_nodes=nodes, trace_capacity=0)
    sub = np.unique(np.linspace(0, sysm.n_fibers - 1, min(subset_fibers, sysm.n_fibers)).round().astype(np.int64))
    ssys = WL.subset(sysm, sub)
    sub_nodes = SH.node_index(sysm.fiber_offsets, sub)
    split = S.FastMonodomainSolver(ssys, method="split", precision="fp64", device=device,
                                   trace_nodes=traced_nodes(ssys, per_fiber), trace_capacity=0)
    split.clamp_override = SH.shard_clamp_nodes(sysm, sub, SH.global_clamp_nodes(sysm))
    runs["fp64_split_subset"] = split
    try:
        for r in runs.values():
            r.initialize()
            r.record_activation(threshold, 16)
            r.reset_timing()
        n_chunks = max(1, int(round(span_ms / chunk_ms)))
        err32 = np.zeros(n_chunks)
        err_split = np.zeros(n_chunks)
        t = 0.0
        for c in range(n_chunks):
            t1 = span_ms if c == n_chunks - 1 else (c + 1) * chunk_ms
            for r in runs.values():
                r.setTimeSpan(t, t1)
                r.advanceTimeSpan()
            v64 = runs["fp64_fused"].vm()
            err32[c] = np.max(np.abs(runs["fp32_fused"].vm() - v64))
            err_split[c] = np.max(np.abs(runs["fp64_split_subset"].vm() - v64[sub_nodes]))
            t = t1
        vm_range = [float(v64.min()), float(v64.max())]
        act = {k: r.activation_steps() for k, r in runs.items()}
        steps = {k: r.split_steps() for k, r in runs.items()}
        rate = {k: r.system.n_nodes * steps[k] / (r.timing()["advance_ms"] / 1e3) for k, r in runs.items()}
        layouts = {k: runs[k].fused_layout() for k in ("fp32_fused", "fp64_fused")}
    finally:
        for r in runs.values():
            r.close()
    sel = np.concatenate([np.arange(f * per_fiber, (f + 1) * per_fiber) for f in sub])
    return {"workload": "%d fibers (%d nodes), %g ms (%d Strang steps); Vm of every node compared after every "
                        "%g ms" % (sysm.n_fibers, sysm.n_nodes, span_ms, steps["fp32_fused"], chunk_ms),
            "fp32_fused_vs_fp64_fused": {
                "vm_max_abs_diff_mV": float(err32.max()),
                "vm_max_abs_diff_mV_per_10_chunks": [float(err32[i:i + 10].max()) for i in range(0, n_chunks, 10)],
                "activation": compare_activation(*act["fp32_fused"], *act["fp64_fused"])},
            "fp64_split_vs_fp64_fused": {
                "fibers": int(len(sub)), "nodes": int(ssys.n_nodes), "vm_max_abs_diff_mV": float(err_split.max()),
                "activation": compare_activation(act["fp64_split_subset"][0], act["fp64_split_subset"][1],
                                                 act["fp64_fused"][0][sel], act["fp64_fused"][1][sel])},
            "vm_range_fp64_mV": vm_range, "activation_threshold_mV": threshold, "dt_split_ms": sysm.dt_splitting,
            "node_steps_per_s": {k: float(v) for k, v in rate.items()}, "fused_layouts": layouts}
