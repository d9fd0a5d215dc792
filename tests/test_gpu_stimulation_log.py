"""Stimulation log (the reference's StimulationLogging, fed at fast_monodomain_solver_compute.tpp:603-607): the
stimulation begins the device records equal the oracle's, time for time."""
import numpy as np
import pytest

import helpers as H
from oracle import oracle as O
from opendihu_b200 import output
from opendihu_b200 import solver as S

pytestmark = pytest.mark.gpu


def _system(rule="vc"):
    # 5 fibers, uneven lengths, check frequency 0.4/ms with jitter, seeded firing tables over 3 motor units,
    # one fiber enabled late
    rng = np.random.default_rng(7)
    s = S.uniform_fibers(H.HH, [121, 97, 160, 88, 133], 0.01, 3.828 / 500, call_frequency=0.4,
                         repeat_after_first_call=0.3, call_enable_begin=0.0, end_time=12.0, dt_0d=1e-4,
                         dt_1d=1e-3, dt_splitting=1e-3, dt_repeated_call=1e-3)
    s.firing_events = (rng.random((20, 3)) < 0.6).astype(np.uint8)
    s.motor_unit_no = np.array([0, 1, 2, 1, 0], np.int32)
    s.jitter = rng.uniform(-0.1, 0.1, (5, 3))
    s.call_enable_begin = np.array([0.0, 0.0, 1.2, 0.0, 0.35])
    s.clamp_rule = rule
    return H.complete(s)


def _oracle_log(s):
    spec = H.oracle_spec(s.copy(), n_threads=2)
    spec["log_capacity"] = 10000
    run = O.OracleRun(spec)
    st = np.ascontiguousarray(s.states, np.float64).copy()
    run.run(st)
    t, f, lost = run.stimulation_log()
    assert lost == 0
    order = np.lexsort((f, t))
    return t[order], f[order]


@pytest.mark.parametrize("method,precision,rule", [("split", "fp64", "vc"), ("fused", "fp32", "vc"),
                                                   ("split", "fp64", "center")])
def test_stimulation_log_equals_oracle(method, precision, rule):
    s = _system(rule)
    t_ref, f_ref = _oracle_log(s)
    assert len(t_ref) >= 10 and len(set(f_ref.tolist())) >= 4
    with S.FastMonodomainSolver(s.copy(), method=method, precision=precision, steps_per_launch=100) as slv:
        slv.enable_stimulation_log(capacity=1)        # grows before the advance
        slv.advanceTimeSpan()
        log = slv.stimulation_log()
    np.testing.assert_array_equal(log["time"], t_ref)          # bit for bit: the same time arithmetic
    np.testing.assert_array_equal(log["fiber"], f_ref)
    np.testing.assert_array_equal(log["motorUnit"], s.motor_unit_no[f_ref])
    # over two advances the log continues across the boundary (the pieces of the second span start from its
    # own start time, so the times agree to rounding)
    with S.FastMonodomainSolver(s.copy(), method=method, precision=precision, steps_per_launch=100) as slv:
        slv.enable_stimulation_log()
        slv.setTimeSpan(0.0, 5.0)
        slv.advanceTimeSpan()
        slv.setTimeSpan(5.0, 12.0)
        slv.advanceTimeSpan()
        log2 = slv.stimulation_log()
    np.testing.assert_array_equal(log2["fiber"], f_ref)
    np.testing.assert_allclose(log2["time"], t_ref, rtol=0, atol=1e-12)


def test_stimulation_log_file_from_settings(tmp_path):
    from test_only_if_stimulated import reference_settings
    (tmp_path / "fd.txt").write_text("1 2")
    (tmp_path / "ft.txt").write_text("1 1\n1 1\n")
    cfg = reference_settings(n_fibers=2, n_elements=30, onlyComputeIfHasBeenStimulated=False,
                             disableComputationWhenStatesAreCloseToEquilibrium=False,
                             fiberDistributionFile="fd.txt", firingTimesFile="ft.txt")
    cfg["RepeatedCall"]["endTime"] = 25.0
    strang = cfg["RepeatedCall"]["MultipleInstances"]["instances"][0]["StrangSplitting"]
    for i, inst in enumerate(strang["Term1"]["MultipleInstances"]["instances"]):
        inst["Heun"]["CellML"]["stimulationLogFilename"] = str(tmp_path / "out" / "stimulation.log")
        inst["Heun"]["CellML"]["additionalArgument"] = 10 + i
    s = S.parse_settings(cfg, base_dir=str(tmp_path))
    assert list(s.fiber_numbers) == [10, 11]
    slv = S.FastMonodomainSolver(s, method="split", precision="fp64")
    slv.run()
    log = slv.stimulation_log()
    slv.close()                                   # the log file is written when the solver closes
    text = (tmp_path / "out" / "stimulation.log").read_text()
    lines = text.split("\n")
    assert lines[0] == "# motor unit no; fiber no; stimulation times in ms"
    # every 10 ms from t = 0: three begins per fiber, fibers numbered by additionalArgument
    np.testing.assert_array_equal(np.unique(log["fiber"]), [10, 11])
    assert len(log["time"]) == 6
    expect = [f"{m};{f};" + "".join(f"{t:g};" for t in log["time"][log["fiber"] == f])
              for m, f in sorted({(int(m), int(f)) for m, f in zip(log["motorUnit"], log["fiber"])})]
    assert lines[1:] == expect


@pytest.mark.parametrize("method,precision", [("split", "fp64"), ("fused", "fp32")])
def test_stimulation_log_over_async_advances_equals_oracle(method, precision):
    """advance_async grows the log before it enqueues, as the blocking advance does: two asynchronous advances
    from a capacity of one entry record every begin of the oracle."""
    s = _system()
    t_ref, f_ref = _oracle_log(s)
    with S.FastMonodomainSolver(s.copy(), method=method, precision=precision, steps_per_launch=100) as slv:
        slv.enable_stimulation_log(capacity=1)
        slv._call(S.N.lib().fdm_set_stimulation_log, 1)   # shrink back to one entry: the growth must come
        slv.setTimeSpan(0.0, 5.0)                           # from the asynchronous advances themselves
        slv.advance_async()
        slv.wait()
        slv.setTimeSpan(5.0, 12.0)
        slv.advance_async()
        slv.wait()
        log = slv.stimulation_log()
    np.testing.assert_array_equal(log["fiber"], f_ref)
    np.testing.assert_allclose(log["time"], t_ref, rtol=0, atol=1e-12)


def test_stimulation_log_never_returns_an_incomplete_log():
    """A capacity too small for the span (the growth before the advance bypassed): the count still counts every
    begin, but reading the entries fails loudly instead of returning unwritten records."""
    import ctypes as C
    s = _system()
    t_ref, _ = _oracle_log(s)
    L = S.N.lib()
    with S.FastMonodomainSolver(s.copy(), method="split", precision="fp64", steps_per_launch=100) as slv:
        slv.initialize()
        slv._call(L.fdm_set_stimulation_log, 3)
        slv._call(L.fdm_advance, 0.0, 12.0)            # the C ABI directly: no growth before the advance
        n = C.c_int64()
        slv._call(L.fdm_get_stimulation_log, C.byref(n), None, None)
        assert n.value == len(t_ref)
        with pytest.raises(RuntimeError, match="incomplete"):
            slv.stimulation_log()
        # growing the log afterwards keeps the three stored entries and the dropped count
        slv._call(L.fdm_set_stimulation_log, 1000)
        slv._call(L.fdm_get_stimulation_log, C.byref(n), None, None)
        assert n.value == len(t_ref)
        with pytest.raises(RuntimeError, match="incomplete"):
            slv.stimulation_log()
