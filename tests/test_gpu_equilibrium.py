"""disableComputationWhenStatesAreCloseToEquilibrium on the GPU (split path) against the oracle's literal
restatement of the reference's buffer walk (compute.tpp:130-265, 630-797): Vm and states, every buffer's
status and the per-rank counts (the counts drift as the reference's do), with and without
onlyComputeIfHasBeenStimulated, several ranks and lane widths, padding lanes, Crank-Nicolson."""
import numpy as np
import pytest

import helpers as H
import test_gpu_parity as GP
from oracle import oracle as O
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL

pytestmark = pytest.mark.gpu

_REST = None


def _rest():
    global _REST
    if _REST is None:
        ns, na, npar, init = O.model_info(H.HH)
        _REST = O.explicit_euler_cell(H.HH, init, np.array([0.0, 120.0, 36.0]), 1e-4, 1000000)
    return _REST


def _system(at_rest=True, only=False, n_ranks=1, width=4, scheme="ImplicitEuler", end_time=2.0, seed=5):
    s = WL.batched_hh(clamp_rule="vc", n_fibers=5, min_nodes=30, max_nodes=61, seed=seed, end_time=end_time,
                      diffusion_scheme=scheme, n_ranks=n_ranks, vc_width=width)
    s.firing_events = np.array([[1, 0, 1, 1, 0]], np.uint8)
    s.motor_unit_no = np.arange(5, dtype=np.int32)
    s.call_enable_begin = np.array([0.0, 0.0, 0.6, 1.2345, 0.0])
    H.complete(s)
    if at_rest:
        s.states = np.repeat(_rest()[:, None], s.n_nodes, axis=1)
    s.skip_close_to_equilibrium = True
    s.only_compute_if_has_been_stimulated = only
    return s


def _oracle(system):
    spec = H.oracle_spec(system.copy())
    run = O.OracleRun(spec)
    st = np.ascontiguousarray(system.states, np.float64).copy()
    n = run.run(st)
    return st, run.eq_status.copy(), run.eq_counter.copy(), n


@pytest.mark.parametrize("at_rest,only,n_ranks,width,scheme", [
    (True, False, 1, 4, "ImplicitEuler"),
    (True, True, 1, 4, "CrankNicolson"),
    (True, False, 2, 4, "ImplicitEuler"),
    (False, False, 1, 4, "ImplicitEuler"),      # initial values off equilibrium: padding lanes keep moving
    (True, True, 3, 8, "ImplicitEuler"),
])
def test_matches_oracle(at_rest, only, n_ranks, width, scheme):
    s = _system(at_rest, only, n_ranks, width, scheme)
    ref, ref_status, ref_counter, n_ref = _oracle(s)
    with S.FastMonodomainSolver(s.copy(), method="split", precision="fp64") as slv:
        slv.advanceTimeSpan()
        st = slv.states()
        status, counter = slv.equilibrium_state()
        assert slv.split_steps() == n_ref
    assert np.max(np.abs(st[0] - ref[0])) <= GP.VM_TOL_FP64
    assert np.max(np.abs(st[1:] - ref[1:])) <= 1e-8
    np.testing.assert_array_equal(status, ref_status)
    np.testing.assert_array_equal(counter, ref_counter)
    if at_rest:
        assert np.any(status == 0)   # buffers at rest were skipped


def test_repeated_advances_and_checkpoint():
    s = _system(end_time=1.6)
    ref, ref_status, ref_counter, _ = _oracle(s)
    with S.FastMonodomainSolver(s.copy(), method="split", precision="fp64", steps_per_launch=37) as slv:
        slv.setTimeSpan(0.0, 0.7)
        slv.advanceTimeSpan()
        slv.saveFiberDataCheckpoint()
        slv.setTimeSpan(0.7, 1.6)
        slv.advanceTimeSpan()
        a = slv.states()
        sa, ca = slv.equilibrium_state()
        slv.restoreFiberDataCheckpoint()
        slv.advanceTimeSpan()
        b = slv.states()
        sb, cb = slv.equilibrium_state()
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(sa, sb)
    np.testing.assert_array_equal(ca, cb)
    assert np.max(np.abs(a[0] - ref[0])) <= GP.VM_TOL_FP64
    np.testing.assert_array_equal(sa, ref_status)
    np.testing.assert_array_equal(ca, ref_counter)


def test_unsupported_combinations_fail_loudly():
    s = _system()
    with pytest.raises(S.N.FdmError):
        S.FastMonodomainSolver(s.copy(), method="fused", precision="fp32").initialize()
    s.clamp_rule = "center"
    with pytest.raises(S.N.FdmError):
        S.FastMonodomainSolver(s.copy(), method="split").initialize()


def _state_information(system, status, has_been_stimulated):
    """computeStateInformation per node as communication.tpp:249-290 forms it: the status of the point buffer
    (valuesOffset + valueNo) / W of the rank that computes the fiber (fiber % nRanks), -1 on a fiber not
    stimulated yet under onlyComputeIfHasBeenStimulated."""
    off = np.asarray(system.fiber_offsets)
    lengths = np.diff(off)
    W, R = system.vc_width, system.n_ranks
    first = np.concatenate([[0], np.cumsum([(lengths[r::R].sum() + W - 1) // W for r in range(R)])])
    out = np.empty(system.n_nodes)
    offset = np.zeros(R, np.int64)
    for f in range(system.n_fibers):
        r = f % R
        buf = first[r] + (offset[r] + np.arange(lengths[f])) // W
        out[off[f]:off[f + 1]] = status[buf]
        if system.only_compute_if_has_been_stimulated and not has_been_stimulated[f]:
            out[off[f]:off[f + 1]] = -1.0
        offset[r] += lengths[f]
    return out


@pytest.mark.parametrize("skip,only,n_ranks,width", [(True, False, 1, 4), (True, True, 3, 8), (False, True, 2, 4),
                                                     (False, False, 1, 4)])
def test_compute_state_information(skip, only, n_ranks, width):
    s = _system(True, only, n_ranks, width, end_time=1.0)
    s.skip_close_to_equilibrium = skip
    s.compute_state_information = True
    run = O.OracleRun(H.oracle_spec(s.copy()))
    st = np.ascontiguousarray(s.states, np.float64).copy()
    run.run(st)
    want = _state_information(s, run.eq_status, run.has_been_stimulated)
    with S.FastMonodomainSolver(s.copy(), method="split", precision="fp64") as slv:
        slv.advanceTimeSpan()
        got = slv.data()["computeStateInformation"]
    np.testing.assert_array_equal(got, want)
    if skip and n_ranks == 1:
        assert np.any(got == 0)       # buffers at rest were counted inactive
    if only:
        assert np.any(got == -1)      # fiber 3 starts at 1.2345 ms


def test_many_fibers_warp_diffusion_with_the_skip():
    # 600 fibers: the split path's diffusion takes a warp per fiber and skips the ranks counted at rest
    s = WL.batched_hh(clamp_rule="vc", n_fibers=600, min_nodes=8, max_nodes=24, seed=7, end_time=0.6, n_ranks=2)
    s.firing_events = np.zeros((1, 100), np.uint8)
    s.firing_events[0, :3] = 1
    H.complete(s)
    s.states = np.repeat(_rest()[:, None], s.n_nodes, axis=1)
    s.skip_close_to_equilibrium = True
    ref, ref_status, ref_counter, _ = _oracle(s)
    with S.FastMonodomainSolver(s.copy(), method="split", precision="fp64") as slv:
        slv.advanceTimeSpan()
        st = slv.states()
        status, counter = slv.equilibrium_state()
    assert np.max(np.abs(st[0] - ref[0])) <= GP.VM_TOL_FP64
    np.testing.assert_array_equal(status, ref_status)
    np.testing.assert_array_equal(counter, ref_counter)
