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
    s = WL.batched_hh(n_fibers=5, min_nodes=30, max_nodes=61, seed=seed, end_time=end_time,
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
