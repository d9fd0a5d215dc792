"""PythonFile-compatible output: written files load with the reference's own reader where it is available
(testing/unit_testing/src/py_reader.py, imported from the reference checkout in this container only)."""
import importlib.util
import os

import numpy as np
import pytest

import helpers as H
from opendihu_b200 import output

#: the reference's reader, where a run names the checkout ($OPENDIHU_REFERENCE); skipped otherwise
REF = os.environ.get("OPENDIHU_REFERENCE", "")
REF_READER = os.path.join(REF, "testing/unit_testing/src/py_reader.py") if REF else ""


@pytest.mark.parametrize("binary", [False, True])
def test_write_and_read_fibers(tmp_path, binary):
    sysm = H.c1_system(n_fibers=2, n_nodes=11, end_time=0.0)
    H.complete(sysm)
    st = sysm.states.copy()
    st[0] += np.arange(22)
    names = ["membrane/V", "sodium_channel_m_gate/m", "sodium_channel_h_gate/h", "potassium_channel_n_gate/n"]
    info = np.where(np.arange(22) < 11, 2.0, -1.0)
    paths = output.write_fibers(str(tmp_path / "fibers"), 9, sysm, st, names, states_for_transfer=[0, 1],
                                time_step_no=90001, current_time=0.90001, binary=binary,
                                additional={"computeStateInformation": info})
    assert len(paths) == 2 and paths[1].endswith("fibers_1_0000009.py")
    d = output.read(paths[1])
    comps = {c["name"]: c["values"] for c in d["data"][1]["components"]}
    np.testing.assert_array_equal(comps["membrane/V"], st[0, 11:22])
    np.testing.assert_allclose(d["data"][0]["components"][0]["values"][-1], 0.1)
    assert d["timeStepNo"] == 90001 and d["nElementsGlobal"] == [10]
    assert d["data"][2]["name"] == "computeStateInformation" and d["data"][2]["components"][0]["values"] == [-1.0] * 11
    if os.path.exists(REF_READER):
        spec = importlib.util.spec_from_file_location("py_reader", REF_READER)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        data = mod.load_data([paths[0]])
        vals = mod.get_values(data[0], "solution", "membrane/V")
        np.testing.assert_array_equal(vals, st[0, :11])
        np.testing.assert_array_equal(mod.get_values(data[0], "computeStateInformation", "0"), info[:11])


def _writes(interval, increments, numbering="incremental", time_step_no=0):
    w = output.OutputWriter({"format": "PythonFile", "outputInterval": interval, "filename": "out/f",
                             "fileNumbering": numbering}, [0])
    return [w.prepare(time_step_no, 0.0, inc) for inc in increments]


def test_output_schedule_follows_the_reference_examples():
    # the two tables in the comment of OutputWriter::Generic::prepareWrite (generic.tpp:34-57): a first call
    # with increment 0 writes the initial values, then every outputInterval-th call writes
    assert [n is not None for n in _writes(2, [0, 1, 1, 1, 1])] == [True, False, True, False, True]
    assert [n is not None for n in _writes(4, [0] + [1] * 8)] == [True] + [False] * 3 + [True] + [False] * 3 + [True]
    # incremental numbering counts the files, timeStepIndex uses the call counter
    assert [n for n in _writes(2, [0, 1, 1, 1, 1]) if n] == ["out/f_0000000", "out/f_0000001", "out/f_0000002"]
    assert [n for n in _writes(2, [0, 1, 1, 1, 1], "timeStepIndex") if n] == \
        ["out/f_0000000", "out/f_0000002", "out/f_0000004"]
    # a call whose increment passes a multiple writes once (several split steps per RepeatedCall piece)
    assert [n is not None for n in _writes(3, [5, 5, 5, 5])] == [True, True, True, True]
    assert [n is not None for n in _writes(10, [3] * 8)] == [False, False, False, True, False, False, True, False]
    # timeStepNo -1: no number in the name
    assert _writes(1, [1], time_step_no=-1) == ["out/f"]
    # outputInterval is read as an int and must be positive (generic.cpp:20)
    w = output.OutputWriter({"format": "PythonFile", "outputInterval": 12.9}, [0])
    assert w.output_interval == 12
    assert output.OutputWriter({"format": "PythonFile", "outputInterval": 0}, [0]).output_interval == 1


def test_output_formats(tmp_path):
    d0 = output.fiber_dict({"0": np.arange(3.0)}, None, 0, 0.5)
    d1 = output.fiber_dict({"0": np.arange(4.0)}, None, 0, 0.5)
    w = output.OutputWriter({"format": "PythonFile", "filename": str(tmp_path / "a" / "fiber"), "binary": True},
                            [3])
    name = w.prepare(0, 0.5, 1)
    paths = w.write(name, [d0])
    assert paths == [str(tmp_path / "a" / "fiber_0000000.py")]
    assert output.read(paths[0])["data"][1]["components"][0]["values"] == [0.0, 1.0, 2.0]
    # a writer over several fibers writes one file per fiber mesh (python_file.tpp:30-43)
    w = output.OutputWriter({"format": "PythonFile", "filename": str(tmp_path / "all")}, [0, 1],
                            ["MeshFiber_0", "MeshFiber_1"])
    paths = w.write(w.prepare(0, 0.5, 1), [d0, d1])
    assert [os.path.basename(p) for p in paths] == ["all_0000000_MeshFiber_0.py", "all_0000000_MeshFiber_1.py"]
    got = []
    w = output.OutputWriter({"format": "PythonCallback", "callback": got.append, "outputInterval": 2}, [0, 1])
    for _ in range(4):
        name = w.prepare(0, 0.5, 1)
        if name:
            w.write(name, [d0, d1])
    assert len(got) == 2 and len(got[0]) == 2 and got[0][1]["currentTime"] == 0.5
    with pytest.warns(UserWarning, match="not built"):
        w = output.OutputWriter({"format": "Paraview"}, [0])
    assert w.write(w.prepare(0, 0.5, 1), [d0]) == []
    with pytest.raises(ValueError):
        output.OutputWriter({"format": "PythonCallback"}, [0])


def test_output_writers_from_settings():
    from test_only_if_stimulated import reference_settings
    from opendihu_b200 import solver as S
    cfg = reference_settings(n_fibers=3)
    term2 = cfg["RepeatedCall"]["MultipleInstances"]["instances"][0]["StrangSplitting"]["Term2"]["MultipleInstances"]
    for i, inst in enumerate(term2["instances"]):
        inst["ImplicitEuler"]["OutputWriter"] = [{"format": "PythonFile", "filename": f"out/fiber_{i}"}]
        inst["ImplicitEuler"]["nAdditionalFieldVariables"] = 2
    term2["OutputWriter"] = [{"format": "PythonFile", "filename": "out/all", "outputInterval": 5}]
    s = S.parse_settings(cfg)
    assert [(w["filename"], f) for w, f in s.output_writers] == \
        [("out/fiber_0", [0]), ("out/fiber_1", [1]), ("out/fiber_2", [2]), ("out/all", [0, 1, 2])]
    assert s.n_additional_field_variables == 2
    term2["OutputWriter"] = None          # the examples set the list to None when output is off
    for inst in term2["instances"]:
        inst["ImplicitEuler"].pop("OutputWriter")
    assert S.parse_settings(cfg).output_writers == []


def test_stimulation_log_format(tmp_path):
    # StimulationLogging::writeLogFile (stimulation_logging.cpp:119-165): sorted by motor unit, fiber, time;
    # one line per (motor unit, fiber), times as a C++ stream writes doubles, no newline at the end
    path = str(tmp_path / "log" / "stimulation.log")
    output.write_stimulation_log(path, [10.0, 0.0, 5e-05, 20.0, 0.123456789], [3, 3, 1, 3, 1], [2, 2, 0, 2, 0])
    assert open(path).read() == ("# motor unit no; fiber no; stimulation times in ms\n"
                                 "0;1;5e-05;0.123457;\n2;3;0;10;20;")
    output.write_stimulation_log(str(tmp_path / "empty.log"), [], [], [])
    assert not os.path.exists(str(tmp_path / "empty.log"))
