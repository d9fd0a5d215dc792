"""Failure detection and recovery, with every failure made on the host (no GPU fault, trap or hang):

* an allocation that fails (the library's fdm_debug_fail_allocation hook) at each allocation of a solver's
  life in turn: the call that meets it fails with FDM_ERR_CUDA and a message, the solver is destroyed cleanly,
  and the library keeps working (a later run is bit-identical to one that never failed);
* a failed fdm_set_fibers on a live solver, repeated with the hook off: the same handle runs on, bit-identical;
* an advance aborted by a corrupt input (a NaN written into Vm, caught by the non-finite check), then
  restoreFiberDataCheckpoint (fast_monodomain_solver_communication.tpp:497-509) and the advance again: the
  result is bit-identical to the run that never failed;
* a wait with a limit (fdm_wait_for) that gives up on a running advance with FDM_ERR_TIMEOUT and leaves it
  enqueued; the later wait completes it with the blocking call's result.

The reference fails loudly on such conditions (LOG(FATAL), fast_monodomain_solver_gpu.tpp:201-205); here every
one is a status code and a message, and the process carries on.
"""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from opendihu_b200 import _native as N
from opendihu_b200 import solver as S

pytestmark = pytest.mark.gpu


def _system():
    s = H.c1_system(n_fibers=3, n_nodes=151, end_time=2.0)
    return H.complete(s)


def _run(system, method, precision, with_checkpoint=True):
    with S.FastMonodomainSolver(system.copy(), method=method, precision=precision, steps_per_launch=50) as slv:
        slv.setTimeSpan(0.0, 1.0)
        slv.advanceTimeSpan()
        if with_checkpoint:
            slv.saveFiberDataCheckpoint()
        slv.setTimeSpan(1.0, 2.0)
        slv.advanceTimeSpan()
        return slv.states()


@pytest.fixture
def no_injection():
    yield
    N.check(N.lib().fdm_debug_fail_allocation(0))


@pytest.mark.parametrize("method,precision", [("split", "fp64"), ("fused", "fp32")])
def test_every_allocation_failure_is_reported_and_cleaned_up(method, precision, no_injection):
    system = _system()
    ref = _run(system, method, precision)
    failures = 0
    for k in range(1, 200):
        N.check(N.lib().fdm_debug_fail_allocation(k))
        try:
            _run(system, method, precision)
        except N.FdmError as e:
            assert e.code == N.FDM_ERR_CUDA, str(e)
            assert "out of memory" in str(e), str(e)
            failures += 1
            continue
        finally:
            N.check(N.lib().fdm_debug_fail_allocation(0))
        break              # the k-th allocation never came: every earlier one has been failed once
    else:
        pytest.fail("more than 199 allocations in one small run")
    assert failures >= 10, failures
    # the library is intact: the same run again, bit for bit
    again = _run(system, method, precision)
    assert np.array_equal(again.view(np.int64), ref.view(np.int64))


def test_failed_set_fibers_leaves_a_usable_handle(no_injection):
    system = _system()
    ref = _run(system, "split", "fp64", with_checkpoint=False)
    L = N.lib()
    s = system.copy()
    with S.FastMonodomainSolver(s, method="split", precision="fp64", steps_per_launch=50) as slv:
        slv.initialize()
        off = np.ascontiguousarray(s.fiber_offsets, np.int64)
        elem = np.ascontiguousarray(s.element_lengths, np.float64)
        pf = np.ascontiguousarray(s.prefactor, np.float64)
        args = (len(off) - 1, N.ptr(off, C.c_int64), N.ptr(elem, C.c_double), N.ptr(pf, C.c_double))
        # a larger fiber set needs larger buffers: the first reallocation fails
        big = np.concatenate([off, off[-1] + off[1:]])
        big_elem = np.concatenate([elem, elem])
        big_pf = np.concatenate([pf, pf])
        N.check(L.fdm_debug_fail_allocation(1))
        rc = L.fdm_set_fibers(slv._h, len(big) - 1, N.ptr(big, C.c_int64), N.ptr(big_elem, C.c_double),
                              N.ptr(big_pf, C.c_double))
        N.check(L.fdm_debug_fail_allocation(0))
        assert rc == N.FDM_ERR_CUDA
        assert b"out of memory" in L.fdm_last_error(slv._h)
        # the solver now holds no fibers: an advance has nothing to do and fails nothing
        slv._call(L.fdm_advance, 0.0, 0.01)
        # the same handle, configured again
        slv._call(L.fdm_set_fibers, *args)
        p = np.ascontiguousarray(s.parameters, np.float64)
        slv._call(L.fdm_set_parameters, N.ptr(p, C.c_double))
        st = np.ascontiguousarray(s.states, np.float64)
        slv._call(L.fdm_set_states, N.ptr(st, C.c_double))
        slv._set_stimulation()
        slv._call(L.fdm_advance, 0.0, 1.0)
        slv._call(L.fdm_advance, 1.0, 2.0)
        out = slv.states()
    assert np.array_equal(out.view(np.int64), ref.view(np.int64))


@pytest.mark.parametrize("method,precision", [("split", "fp64"), ("fused", "fp32")])
def test_aborted_advance_resumes_from_checkpoint_bit_identical(method, precision):
    system = _system()
    ref = _run(system, method, precision)
    with S.FastMonodomainSolver(system.copy(), method=method, precision=precision, steps_per_launch=50) as slv:
        slv.setTimeSpan(0.0, 1.0)
        slv.advanceTimeSpan()
        slv.saveFiberDataCheckpoint()
        bad = slv.states()
        bad[0, 200] = np.nan                      # a corrupt input
        slv.set_states(bad)
        slv.setTimeSpan(1.0, 2.0)
        with pytest.raises(N.FdmError) as ei:
            slv.advanceTimeSpan()
        assert ei.value.code == N.FDM_ERR_NAN
        slv.restoreFiberDataCheckpoint()
        slv.advanceTimeSpan()
        out = slv.states()
    assert np.array_equal(out.view(np.int64), ref.view(np.int64))


def test_wait_with_a_limit_gives_up_and_the_advance_completes_later():
    system = H.complete(H.c1_system(n_fibers=64, n_nodes=1481, end_time=3.0))
    with S.FastMonodomainSolver(system.copy(), method="split", precision="fp64") as slv:
        slv.setTimeSpan(0.0, 3.0)
        slv.advanceTimeSpan()
        ref = slv.states()
    with S.FastMonodomainSolver(system.copy(), method="split", precision="fp64") as slv:
        slv.setTimeSpan(0.0, 3.0)
        slv.advance_async()
        assert slv.wait_for(0.0) is False          # the last window of 3000 Strang steps is still running
        assert slv.wait_for(120.0) is True
        assert slv.wait_for(0.0) is True           # nothing pending any more
        out = slv.states()
    assert np.array_equal(out.view(np.int64), ref.view(np.int64))


def test_wait_for_rejects_a_negative_limit():
    system = _system()
    with S.FastMonodomainSolver(system.copy(), method="split", precision="fp64") as slv:
        slv.initialize()
        assert N.lib().fdm_wait_for(slv._h, -1.0) == N.FDM_ERR_ARG
