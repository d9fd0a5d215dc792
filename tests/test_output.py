"""PythonFile-compatible output: written files load with the reference's own reader where it is available
(testing/unit_testing/src/py_reader.py, imported from the reference checkout in this container only)."""
import importlib.util
import os

import numpy as np
import pytest

import helpers as H
from opendihu_b200 import output

REF_READER = os.path.join(os.environ.get("OPENDIHU_REFERENCE", "/root/reference"), "testing/unit_testing/src/py_reader.py")


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
