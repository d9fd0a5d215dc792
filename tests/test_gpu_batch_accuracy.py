"""Accuracy over the full spans of the benchmark configurations (slow GPU tests).

* Batching + precision configuration, all 4096 fibers over its 100 ms (Poisson firing: several action
  potentials per fiber): the FP32-reaction fused solver within 0.1 mV of the FP64 solver at every node after
  every 1 ms, and its activation steps at 32 nodes per fiber within one split step; the FP64 fused solver equal
  to the FP64 split ("plain") solver on 64 fibers of the batch to 1e-6 mV with identical activation steps.
* The FP64 split solver against the CPU oracle on the shortest fibers of that batch over the same 100 ms:
  Vm to 1e-6 mV and identical activation steps at 32 nodes per fiber (OPENDIHU_ORACLE_FIBERS fibers, 64 by
  default; the oracle runs on all host cores, about 3 minutes on 16).
* Shorten 2007 (56 states) over 2 ms with an action potential: split FP64 against the oracle to 1e-6 mV, the
  FP32 reaction within 0.1 mV.
"""
import os

import numpy as np
import pytest

import helpers as H
from opendihu_b200 import accuracy as ACC
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

VM_TOL_FP64 = 1e-6
VM_TOL_FP32 = 0.1


def test_batch_fp32_fused_within_01mV_and_one_step_over_100ms():
    res = ACC.batch_accuracy(WL.batched_hh(n_fibers=4096, seed=0), device=0, span_ms=100.0)
    print(res)
    a32 = res["fp32_fused_vs_fp64_fused"]
    assert a32["vm_max_abs_diff_mV"] <= VM_TOL_FP32, a32
    act = a32["activation"]
    assert act["traced_nodes"] == 4096 * 32
    assert act["crossings"] >= 4096 * 32 // 2     # action potentials reach most of the traced nodes
    assert act["nodes_count_mismatch"] == 0 and act["max_step_diff"] <= 1, act
    a64 = res["fp64_split_vs_fp64_fused"]
    assert a64["vm_max_abs_diff_mV"] <= VM_TOL_FP64, a64
    assert a64["activation"]["nodes_count_mismatch"] == 0 and a64["activation"]["max_step_diff"] == 0, a64


def test_fp64_split_equals_oracle_over_the_batch_span():
    n_fibers = int(os.environ.get("OPENDIHU_ORACLE_FIBERS", "64"))
    system = WL.batched_hh(n_fibers=4096, seed=0)
    lengths = np.diff(np.asarray(system.fiber_offsets))
    pick = np.sort(np.argsort(lengths, kind="stable")[:n_fibers])   # the shortest fibers: bounded CPU time
    sub = WL.subset(system, pick)
    sub.start_time, sub.end_time = 0.0, 100.0
    H.complete(sub)
    nodes = ACC.traced_nodes(sub, 32)
    ref, _, tr, n = H.run_oracle(sub.copy(), trace_nodes=nodes, trace_capacity=100000)
    up = (tr[:-1] <= 0.0) & (tr[1:] > 0.0)
    ref_counts = up.sum(axis=0).astype(np.int32)
    ref_steps = np.full((len(nodes), 16), -1, np.int64)
    for k in range(len(nodes)):
        rows = np.nonzero(up[:, k])[0][:16] + 1
        ref_steps[k, :len(rows)] = rows
    with S.FastMonodomainSolver(sub.copy(), method="split", precision="fp64", trace_nodes=nodes,
                                trace_capacity=0) as slv:
        slv.record_activation(0.0, 16)
        slv.advanceTimeSpan()
        st = slv.states()
        counts, steps = slv.activation_steps()
        assert slv.split_steps() == n == 100000
    dv = float(np.max(np.abs(st[0] - ref[0])))
    act = ACC.compare_activation(counts, steps, ref_counts, ref_steps)
    print({"fibers": len(pick), "nodes": sub.n_nodes, "vm_max_abs_diff_mV": dv,
           "states_max_abs_diff": float(np.max(np.abs(st - ref))), "activation": act})
    assert dv <= VM_TOL_FP64
    assert act["crossings"] >= len(nodes)
    assert act["nodes_count_mismatch"] == 0 and act["max_step_diff"] == 0, act


def test_shorten_over_2ms_against_oracle():
    sysm = S.uniform_fibers(H.SHORTEN, [121, 97], 0.01, 3.828 / (500 * 0.58), call_frequency=0.1,
                            repeat_after_first_call=0.1, end_time=2.0, dt_0d=1e-5, dt_1d=5e-4, dt_splitting=5e-4,
                            dt_repeated_call=5e-4)
    H.complete(sysm)
    nodes = ACC.traced_nodes(sysm, 8)
    ref, _, tr, n = H.run_oracle(sysm.copy(), trace_nodes=nodes, trace_capacity=4000)
    assert n == 4000
    assert ref[0].max() > 0 or tr.max() > 0                  # an action potential within the span
    at_ref = H.activation_times(tr, 5e-4)
    for precision, tol in (("fp64", VM_TOL_FP64), ("fp32", VM_TOL_FP32)):
        with S.FastMonodomainSolver(sysm.copy(), method="split", precision=precision, trace_nodes=nodes,
                                    trace_capacity=4000) as slv:
            slv.advanceTimeSpan()
            st = slv.states()
            at = H.activation_times(slv.trace(), 5e-4)
        dv = float(np.max(np.abs(st[0] - ref[0])))
        print(precision, dv)
        assert dv <= tol, (precision, dv)
        assert np.array_equal(np.isnan(at), np.isnan(at_ref))
        ok = ~np.isnan(at)
        assert ok.any()
        assert np.all(np.abs(at[ok] - at_ref[ok]) <= 5e-4 + 1e-12)


def test_shorten_at_scale_sample_against_oracle():
    """Shorten at scale (10,000 fibers of U[1000,2500] nodes, 200 motor units): the 4 shortest fibers among
    those whose motor unit fires at t = 0, over 0.5 ms (1000 Strang steps, an action potential under way):
    FP64 split against the oracle to 1e-6 mV, the FP32 reaction within 0.1 mV."""
    system = WL.shorten_scale(end_time=0.5)
    mu = np.asarray(system.motor_unit_no)
    fires0 = np.nonzero(np.asarray(system.firing_events)[0, mu % system.firing_events.shape[1]])[0]
    lengths = np.diff(np.asarray(system.fiber_offsets))[fires0]
    pick = np.sort(fires0[np.argsort(lengths, kind="stable")[:4]])
    sub = WL.subset(system, pick)
    H.complete(sub)
    ref, _, _, n = H.run_oracle(sub.copy())
    assert n == 1000
    assert ref[0].max() > 0.0                                  # depolarised nodes at the end of the span
    for precision, tol in (("fp64", VM_TOL_FP64), ("fp32", VM_TOL_FP32)):
        with S.FastMonodomainSolver(sub.copy(), method="split", precision=precision) as slv:
            slv.advanceTimeSpan()
            st = slv.states()
            assert slv.split_steps() == n
        dv = float(np.max(np.abs(st[0] - ref[0])))
        print({"fibers": pick.tolist(), "nodes": sub.n_nodes, "precision": precision, "vm_max_abs_diff_mV": dv})
        assert dv <= tol, (precision, dv)
