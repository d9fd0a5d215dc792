"""Output writers of the diffusion solver, run after each RepeatedCall piece of advanceTimeSpan as the
reference's FastMonodomainSolver calls them (fast_monodomain_solver_compute.tpp:35-44), with the call
counting of OutputWriter::Generic::prepareWrite (generic.tpp:14-115)."""
import glob
import os

import numpy as np
import pytest

from opendihu_b200 import _native as N
from opendihu_b200 import output
from opendihu_b200 import solver as S
from test_only_if_stimulated import reference_settings

pytestmark = pytest.mark.gpu


def _settings(tmp_path, per_fiber_interval=25, callback=None):
    (tmp_path / "fd.txt").write_text("1 2")
    (tmp_path / "ft.txt").write_text("1 1\n1 1\n")
    cfg = reference_settings(n_fibers=2, n_elements=40, onlyComputeIfHasBeenStimulated=False,
                             disableComputationWhenStatesAreCloseToEquilibrium=False,
                             fiberDistributionFile="fd.txt", firingTimesFile="ft.txt")
    strang = cfg["RepeatedCall"]["MultipleInstances"]["instances"][0]["StrangSplitting"]
    for inst in strang["Term1"]["MultipleInstances"]["instances"]:
        inst["Heun"]["CellML"]["algebraicsForTransfer"] = [4]
    term2 = strang["Term2"]["MultipleInstances"]
    for i, inst in enumerate(term2["instances"]):
        inst["ImplicitEuler"]["nAdditionalFieldVariables"] = 1
        inst["ImplicitEuler"]["OutputWriter"] = [
            {"format": "PythonFile", "outputInterval": per_fiber_interval,
             "filename": str(tmp_path / "out" / f"fiber_{i}"), "binary": False}]
    if callback is not None:
        term2["OutputWriter"] = [{"format": "PythonCallback", "callback": callback, "outputInterval": 40,
                                  "fileNumbering": "timeStepIndex"}]
    return S.parse_settings(cfg, base_dir=str(tmp_path))


def _vm(d):
    return np.asarray(d["data"][1]["components"][0]["values"])


def test_writers_run_at_the_reference_times(tmp_path):
    got = []
    system = _settings(tmp_path, callback=got.append)
    assert system.end_time == pytest.approx(0.1)
    with S.FastMonodomainSolver(system.copy(), method="split", precision="fp64") as a:
        a.advanceTimeSpan()
        vm_a = a.vm()
        alg_a = a.algebraics()
        # a piece range past the last piece is refused
        assert N.lib().fdm_advance_pieces(a._h, 0.0, 0.1, 0, 101) != 0
    # 100 RepeatedCall pieces of one split step: the per-fiber writers (interval 25) write after pieces
    # 25, 50, 75, 100, the callback (interval 40) after pieces 40 and 80
    for i in range(2):
        files = sorted(glob.glob(str(tmp_path / "out" / f"fiber_{i}_*.py")))
        assert [os.path.basename(f) for f in files] == [f"fiber_{i}_{k:07d}.py" for k in range(4)]
        ds = [output.read(f) for f in files]
        np.testing.assert_allclose([d["currentTime"] for d in ds], [0.025, 0.05, 0.075, 0.1], rtol=1e-12)
        assert all(d["timeStepNo"] == 0 for d in ds)
        off = system.fiber_offsets
        # the last file holds the state at the end of the advance
        np.testing.assert_array_equal(_vm(ds[-1]), vm_a[off[i]:off[i + 1]])
        add = ds[-1]["data"][2]
        assert add["name"] == "additionalFieldVariable0"
        np.testing.assert_array_equal(add["components"][0]["values"], alg_a[0, off[i]:off[i + 1]])
        assert ds[-1]["data"][0]["components"][0]["values"][-1] == pytest.approx(0.4)
    assert len(got) == 2 and [len(x) for x in got] == [2, 2]
    np.testing.assert_allclose([x[0]["currentTime"] for x in got], [0.04, 0.08], rtol=1e-12)
    # stopping after the writing pieces leaves the steps those of one advance: the same end state bit for bit
    with S.FastMonodomainSolver(system.copy(), method="split", precision="fp64") as b:
        b.advanceTimeSpan(withOutputWritersEnabled=False)
        np.testing.assert_array_equal(b.vm(), vm_a)
        assert b.split_steps() == 100
    # the file at t = 0.05 holds the state an advance over [0, 0.05] reaches (its piece times are formed
    # from the shorter span, equal to a few ulps)
    first = output.read(str(tmp_path / "out" / "fiber_1_0000001.py"))
    with S.FastMonodomainSolver(system.copy(), method="split", precision="fp64") as c:
        c.setTimeSpan(0.0, 0.05)
        c.advanceTimeSpan(withOutputWritersEnabled=False)
        off = system.fiber_offsets
        np.testing.assert_allclose(_vm(first), c.vm()[off[1]:off[2]], rtol=0, atol=1e-9)
    assert np.ptp(_vm(first)) > 1.0          # the stimulated fiber is not at rest


def test_call_output_writer(tmp_path):
    system = _settings(tmp_path, per_fiber_interval=2)
    with S.FastMonodomainSolver(system.copy(), method="fused", precision="fp32") as d:
        # before any advance the call counts as the initial-values call and writes
        d.callOutputWriter(0, 0.0)
        d0 = output.read(str(tmp_path / "out" / "fiber_0_0000000.py"))
        assert d0["currentTime"] == 0.0
        np.testing.assert_allclose(_vm(d0), d.vm()[:41])
        d.setTimeSpan(0.0, 0.01)
        d.advanceTimeSpan(withOutputWritersEnabled=False)
        assert len(glob.glob(str(tmp_path / "out" / "fiber_0_*.py"))) == 1
        d.callOutputWriter(1, 0.0, 2)           # 1 % 2 != 0: not called
        d.callOutputWriter(0, 0.0)              # call count 1: no multiple of 2 passed
        assert len(glob.glob(str(tmp_path / "out" / "fiber_0_*.py"))) == 1
        d.callOutputWriter(4, 0.0, 2)           # call count 2: writes, at the end of the last piece
        d1 = output.read(str(tmp_path / "out" / "fiber_0_0000001.py"))
        assert d1["currentTime"] == pytest.approx(0.01)
        np.testing.assert_array_equal(_vm(d1), d.vm()[:41])
