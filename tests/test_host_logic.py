"""Host logic of the Python host class without a device: the C ABI is replaced by a recording fake, so the
order and arguments of the library calls that advanceTimeSpan, the output writers, callOutputWriter and the
stimulation log make can be checked on CPU."""
import ctypes as C
import math

import numpy as np
import pytest

import helpers as H
from opendihu_b200 import _native as N
from opendihu_b200 import output
from opendihu_b200 import solver as S


class FakeLib:
    """Every fdm_* call succeeds and is recorded; the RepeatedCall plan follows the library's step-count rule
    (one split step per piece here); Vm counts the pieces advanced so far; the host-only model queries go to
    the real library."""

    def __init__(self, n_nodes, dt_repeated_call, real=None):
        self.real = real
        self.calls = []
        self.n_nodes = n_nodes
        self.dt_rc = dt_repeated_call
        self.pieces_done = 0
        self.log_t = np.zeros(0)
        self.log_f = np.zeros(0, np.int32)
        self.n_of = {}                     # nodes per solver handle (from fdm_set_fibers)
        self.done_of = {}                  # RepeatedCall pieces advanced per solver handle

    def __getattr__(self, name):
        def call(*args):
            self.calls.append((name,) + args[1:])
            return 0
        return call

    def fdm_create(self, cfg, h):
        h._obj.value = 1000 + len(self.n_of)
        self.n_of[h._obj.value] = self.n_nodes
        return 0

    def fdm_set_fibers(self, h, nf, off, elem, pf):
        self.n_of[h.value] = int(np.ctypeslib.as_array(off, (nf + 1,))[-1])
        return 0

    def fdm_last_error(self, h):
        return b"fake"

    def fdm_model_info(self, *args):
        return self.real.fdm_model_info(*args)

    def fdm_model_parameter_defaults(self, *args):
        return self.real.fdm_model_parameter_defaults(*args)

    def fdm_model_equilibrium(self, model, device, approx, params, dt, states, it, inc, dtf):
        y = np.ctypeslib.as_array(states, (4,))
        self.calls.append(("fdm_model_equilibrium", dt, y.copy(), np.ctypeslib.as_array(params, (3,)).copy()))
        y[:] = [-74.99, 0.053, 0.596, 0.318]
        it._obj.value, inc._obj.value, dtf._obj.value = 1000, 9e-6, dt
        return 0

    def fdm_set_states(self, h, st):
        self.calls.append(("fdm_set_states", np.ctypeslib.as_array(st, (4, self.n_of[h.value])).copy()))
        return 0

    def _n(self, t0, t1):
        return max(1, math.ceil((t1 - t0) / self.dt_rc - 0.1))

    def fdm_repeated_call_plan(self, h, t0, t1, n, steps):
        n._obj.value = self._n(t0, t1)
        if steps:
            np.ctypeslib.as_array(steps, (n._obj.value,))[:] = 1
        return 0

    def fdm_advance(self, h, t0, t1):
        self.calls.append(("fdm_advance", t0, t1))
        self.done_of[h.value] = self.done_of.get(h.value, 0) + self._n(t0, t1)
        return 0

    def fdm_advance_pieces(self, h, t0, t1, k0, k1):
        self.calls.append(("fdm_advance_pieces", k0, k1))
        self.done_of[h.value] = self.done_of.get(h.value, 0) + k1 - k0
        return 0

    def fdm_get_vm(self, h, out):
        np.ctypeslib.as_array(out, (self.n_of[h.value],))[:] = self.done_of.get(h.value, 0)
        return 0

    def fdm_get_stimulation_log(self, h, n, t, f):
        n._obj.value = len(self.log_t)
        if t:
            np.ctypeslib.as_array(t, (len(self.log_t),))[:] = self.log_t
        if f:
            np.ctypeslib.as_array(f, (len(self.log_f),))[:] = self.log_f
        return 0


@pytest.fixture
def fake(monkeypatch):
    holder = {}

    real = N.lib()

    def install(system):
        lib = FakeLib(system.n_nodes, system.dt_repeated_call, real)
        monkeypatch.setattr(N, "lib", lambda: lib)
        holder["lib"] = lib
        return lib
    return install


def _system():
    return H.complete(H.c1_system(n_fibers=2, n_nodes=11, end_time=0.01))


def test_writers_split_the_advance_at_the_writing_pieces(fake):
    s = _system()
    a, b = [], []
    s.output_writers = [({"format": "PythonCallback", "callback": a.append, "outputInterval": 3}, [1]),
                        ({"format": "PythonCallback", "callback": b.append, "outputInterval": 4}, [0, 1])]
    lib = fake(s)
    slv = S.FastMonodomainSolver(s)
    slv.advanceTimeSpan()
    # 10 pieces of one split step: writer a after pieces 3, 6, 9, writer b after 4 and 8
    adv = [c[1:] for c in lib.calls if c[0] == "fdm_advance_pieces"]
    assert adv == [(0, 3), (3, 4), (4, 6), (6, 8), (8, 9), (9, 10)]
    assert [len(x) for x in a] == [1, 1, 1] and [len(x) for x in b] == [2, 2]
    np.testing.assert_allclose([x[0]["currentTime"] for x in a], [0.003, 0.006, 0.009], rtol=1e-12)
    # each dict holds the Vm after its piece (the fake's Vm counts the pieces advanced)
    assert [x[0]["data"][1]["components"][0]["values"][0] for x in a] == [3.0, 6.0, 9.0]
    assert [x[1]["data"][1]["components"][0]["values"][0] for x in b] == [4.0, 8.0]
    # writers off: one advance over the span
    lib.calls.clear()
    slv.setTimeSpan(0.01, 0.02)
    slv.advanceTimeSpan(withOutputWritersEnabled=False)
    assert [c for c in lib.calls if c[0].startswith("fdm_advance")] == [("fdm_advance", 0.01, 0.02)]
    assert len(a) == 3
    # callOutputWriter continues the counts with the last piece's single step
    for k in range(3):
        slv.callOutputWriter(k, 0.0)
    assert len(a) == 4 and a[-1][0]["currentTime"] == pytest.approx(0.02)
    slv.close()


def test_call_output_writer_before_any_advance_writes_the_initial_values(fake):
    s = _system()
    got = []
    s.output_writers = [({"format": "PythonCallback", "callback": got.append, "outputInterval": 5}, [0])]
    fake(s)
    slv = S.FastMonodomainSolver(s)
    slv.callOutputWriter(0, 0.0)
    assert len(got) == 1 and got[0][0]["currentTime"] == 0.0
    slv.callOutputWriter(1, 0.0, 2)      # 1 % 2: not called
    assert len(got) == 1
    slv.close()


def test_stimulation_log_enabled_from_settings_and_written_at_close(fake, tmp_path):
    s = _system()
    s.stimulation_log_filename = str(tmp_path / "out" / "stimulation.log")
    s.fiber_numbers = [7, 9]
    s.motor_unit_no = np.array([3, 1], np.int32)
    lib = fake(s)
    lib.log_t = np.array([10.0, 0.0, 0.0, 10.0])
    lib.log_f = np.array([1, 1, 0, 0], np.int32)
    slv = S.FastMonodomainSolver(s)
    slv.initialize()
    caps = [c[1] for c in lib.calls if c[0] == "fdm_set_stimulation_log"]
    # at most one begin per check period 1/f = 10 ms: ceil(0.01 * 0.1) + 2 per fiber, plus a margin
    assert caps == [2 * 3 + 16]
    slv.advanceTimeSpan()
    grow = [c for c in lib.calls if c[0] == "fdm_set_stimulation_log"]
    assert grow[-1][1] == 4 + 2 * 3 + 16           # entries so far + what the span can add
    log = slv.stimulation_log()
    np.testing.assert_array_equal(log["time"], [0.0, 0.0, 10.0, 10.0])
    np.testing.assert_array_equal(log["fiber"], [7, 9, 7, 9])
    np.testing.assert_array_equal(log["motorUnit"], [3, 1, 3, 1])
    slv.close()
    assert (tmp_path / "out" / "stimulation.log").read_text() == \
        "# motor unit no; fiber no; stimulation times in ms\n1;9;0;10;\n3;7;0;10;"
    assert any(c[0] == "fdm_destroy" for c in lib.calls)


def test_states_initialized_to_equilibrium(fake):
    # "initializeStatesToEquilibrium": the search starts from the first node's states and parameters with the
    # settings' time step width, and every node starts from its result
    s = _system()
    s.states[:, 0] = [-70.0, 0.1, 0.5, 0.3]
    s.parameters[1, 0] = 100.0
    s.initialize_states_to_equilibrium = True
    s.equilibrium_dt = 2e-4
    lib = fake(s)
    slv = S.FastMonodomainSolver(s)
    slv.initialize()
    (name, dt, y0, p0), = [c for c in lib.calls if c[0] == "fdm_model_equilibrium"]
    assert dt == 2e-4
    np.testing.assert_array_equal(y0, [-70.0, 0.1, 0.5, 0.3])
    np.testing.assert_array_equal(p0, s.parameters[:, 0])
    (_, st), = [c for c in lib.calls if c[0] == "fdm_set_states"]
    np.testing.assert_array_equal(st, np.repeat(np.array([-74.99, 0.053, 0.596, 0.318])[:, None], s.n_nodes, 1))
    assert slv.equilibrium["iterations"] == 1000
    slv.close()
    slv.initialize()                      # a second initialize keeps the equilibrium states, no new search
    assert len([c for c in lib.calls if c[0] == "fdm_model_equilibrium"]) == 1
    slv.close()


def test_sharded_solver_merges_the_logs_and_searches_the_equilibrium_once(fake, tmp_path):
    from opendihu_b200 import sharding as SH
    s = H.complete(H.c1_system(n_fibers=3, n_nodes=11, end_time=0.01))
    s.stimulation_log_filename = str(tmp_path / "stimulation.log")
    s.initialize_states_to_equilibrium = True
    s.motor_unit_no = np.array([0, 1, 2], np.int32)
    lib = fake(s)
    lib.log_t = np.array([0.0])
    lib.log_f = np.array([0], np.int32)       # every shard reports its first fiber stimulated at t = 0
    sh = SH.ShardedSolver(s, devices=[0], n_shards=2)
    assert all(not sv.system.stimulation_log_filename for sv in sh.shards)
    sh.initialize()
    assert len([c for c in lib.calls if c[0] == "fdm_model_equilibrium"]) == 1
    sets = [c[1] for c in lib.calls if c[0] == "fdm_set_states"]
    assert sorted(x.shape[1] for x in sets) == [11, 22]
    assert all(np.array_equal(x[:, 0], [-74.99, 0.053, 0.596, 0.318]) for x in sets)
    log = sh.stimulation_log()
    first = sorted(int(f[0]) for f in sh.fibers)
    np.testing.assert_array_equal(log["fiber"], first)
    np.testing.assert_array_equal(log["motorUnit"], s.motor_unit_no[first])
    sh.close()
    lines = (tmp_path / "stimulation.log").read_text().split("\n")
    assert lines[1:] == [f"{s.motor_unit_no[f]};{f};0;" for f in first]


def test_sharded_solver_runs_the_writers_over_the_whole_system(fake):
    from opendihu_b200 import sharding as SH
    s = H.complete(H.c1_system(n_fibers=3, n_nodes=11, end_time=0.01))
    got = []
    s.output_writers = [({"format": "PythonCallback", "callback": got.append, "outputInterval": 4}, [0, 1, 2])]
    lib = fake(s)
    sh = SH.ShardedSolver(s, devices=[0], n_shards=2)
    sh.advanceTimeSpan()
    # both shards stop after pieces 4 and 8 and finish the span; the writer sees all three fibers each time
    adv = [c[1:] for c in lib.calls if c[0] == "fdm_advance_pieces"]
    assert sorted(adv) == sorted([(0, 4), (4, 8), (8, 10)] * 2)
    assert [len(x) for x in got] == [3, 3]
    assert [[d["data"][1]["components"][0]["values"][0] for d in x] for x in got] == [[4.0] * 3, [8.0] * 3]
    np.testing.assert_allclose([x[0]["currentTime"] for x in got], [0.004, 0.008], rtol=1e-12)
    # callOutputWriter continues the count with the last piece's step: calls 11 and 12 write at 12
    sh.callOutputWriter(0, 0.0)
    sh.callOutputWriter(0, 0.0)
    assert len(got) == 3 and got[-1][0]["currentTime"] == pytest.approx(0.01)
    # writers off: one advance per shard
    lib.calls.clear()
    sh.setTimeSpan(0.01, 0.02)
    sh.advanceTimeSpan(withOutputWritersEnabled=False)
    assert [c for c in lib.calls if c[0].startswith("fdm_advance")] == [("fdm_advance", 0.01, 0.02)] * 2
    sh.close()
