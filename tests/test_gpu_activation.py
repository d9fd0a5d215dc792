"""Activation recording on the traced nodes (fdm_set_activation_recording) against the oracle's Vm trace: the
Strang steps after which Vm rises above the threshold, per node, equal the crossings of the oracle's trace
(FP64 paths: identical steps; FP32 reaction: within one step).  A trace set in the middle of a run counts its
rows from there."""
import numpy as np
import pytest

import helpers as H
from opendihu_b200 import solver as S

pytestmark = pytest.mark.gpu

THRESHOLD = 0.0


def _system():
    # 3 fibers, uneven lengths, a stimulus every 4 ms (several action potentials per node over 12 ms)
    s = S.uniform_fibers(H.HH, [301, 257, 330], 0.01, 3.828 / 500, call_frequency=0.25,
                         repeat_after_first_call=0.1, call_enable_begin=0.0, end_time=12.0, dt_0d=1e-4,
                         dt_1d=1e-3, dt_splitting=1e-3, dt_repeated_call=1e-3, diffusion_scheme="CrankNicolson")
    return H.complete(s)


def _nodes(s, per_fiber=32):
    out = []
    for f in range(s.n_fibers):
        a, b = s.fiber_offsets[f], s.fiber_offsets[f + 1]
        out += list(np.linspace(a, b - 1, per_fiber).round().astype(np.int64))
    return np.array(out, np.int64)


def _crossings(trace, threshold=THRESHOLD):
    """Per column, the rows r >= 1 with trace[r-1] <= threshold < trace[r]."""
    up = (trace[:-1] <= threshold) & (trace[1:] > threshold)
    return [list(np.nonzero(up[:, k])[0] + 1) for k in range(trace.shape[1])]


@pytest.mark.parametrize("method,precision", [("split", "fp64"), ("fused", "fp64"), ("fused", "fp32")])
def test_activation_steps_equal_oracle_crossings(method, precision):
    s = _system()
    nodes = _nodes(s)
    _, _, tr, n = H.run_oracle(s.copy(), trace_nodes=nodes, trace_capacity=20000)
    ref = _crossings(tr)
    assert sum(len(r) for r in ref) >= len(nodes)       # an action potential reaches every traced node
    with S.FastMonodomainSolver(s.copy(), method=method, precision=precision, trace_nodes=nodes,
                                trace_capacity=0, steps_per_launch=100) as slv:
        slv.record_activation(THRESHOLD, capacity=8)
        slv.advanceTimeSpan()
        counts, steps = slv.activation_steps()
    for k in range(len(nodes)):
        got = list(steps[k, :counts[k]])
        if precision == "fp64":
            assert got == ref[k], (k, got, ref[k])
        else:
            assert len(got) == len(ref[k]), (k, got, ref[k])
            assert np.all(np.abs(np.array(got) - np.array(ref[k])) <= 1), (k, got, ref[k])
    assert np.all(steps[counts == 0] == -1)


def test_trace_set_mid_run_counts_rows_from_there():
    s = _system()
    nodes = _nodes(s, per_fiber=8)
    _, _, tr, n = H.run_oracle(s.copy(), trace_nodes=nodes, trace_capacity=20000)
    with S.FastMonodomainSolver(s.copy(), method="split", precision="fp64") as slv:
        slv.setTimeSpan(0.0, 5.0)
        slv.advanceTimeSpan()
        slv.set_trace(nodes, 7000)
        slv.record_activation(THRESHOLD, capacity=8)
        slv.setTimeSpan(5.0, 12.0)
        slv.advanceTimeSpan()
        got = slv.trace()
        counts, steps = slv.activation_steps()
    assert got.shape == (7000, len(nodes))
    np.testing.assert_allclose(got, tr[5000:12000], rtol=0, atol=1e-9)
    ref = _crossings(tr[5000:12000])
    for k in range(len(nodes)):
        assert list(steps[k, :counts[k]]) == ref[k]
