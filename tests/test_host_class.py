"""The C++ host class fdm::FastMonodomainSolver (include/fdm_b200.hpp): compiled with g++ against the
library; on CPU it builds, reads the settings the Python harness writes and fails loudly without a device;
on the GPU its run (two advances around a checkpoint, the checkpoint replayed) equals the Python operator's
bit for bit and the oracle within the FP64 tolerance."""
import os
import subprocess

import numpy as np
import pytest

import helpers as H
import test_gpu_parity as GP
from opendihu_b200 import solver as S

SRC = os.path.join(H.ROOT, "tests", "cpp", "host_class_main.cpp")
LIBDIR = os.path.join(H.ROOT, "opendihu_b200")


def _build(tmp_path):
    exe = str(tmp_path / "host_class_main")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(H.ROOT, "include"), SRC,
                    "-L", LIBDIR, "-lfdm_b200", "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    return exe


def _system():
    s = GP.small_system(end_time=0.6, algebraics_for_transfer=[0, 4])
    return H.complete(s)


def test_builds_reads_settings_and_fails_loudly_without_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU test runs the class")
    exe = _build(tmp_path)
    cfg = str(tmp_path / "settings.txt")
    S.write_host_settings(_system(), cfg)
    r = subprocess.run([exe, cfg, str(tmp_path / "out.bin"), "0.3"], capture_output=True, text=True)
    assert r.returncode == 2 and "fdm::Error 5" in r.stderr, (r.returncode, r.stderr)
    r = subprocess.run([exe, str(tmp_path / "missing.txt"), "x", "0.3"], capture_output=True, text=True)
    assert r.returncode == 2 and "cannot open" in r.stderr


def test_settings_file_round_trip(tmp_path):
    # what write_host_settings writes from a parsed system is what FiberSettings::load reads (host only)
    exe = _build(tmp_path)
    s = _system()
    s.fiber_numbers = [7, 8, 9]
    s.initialize_states_to_equilibrium = True
    s.equilibrium_dt = 2.5e-4
    cfg = str(tmp_path / "settings.txt")
    S.write_host_settings(s, cfg)
    out = str(tmp_path / "read.txt")
    r = subprocess.run([exe, cfg, out, "0", "settings"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = dict(line.split(" ", 1) for line in open(out).read().splitlines())
    assert got["n_fibers"] == "3" and got["n_nodes"] == str(s.n_nodes)
    assert got["equilibrium"] == "1 0.00025000000000000001"
    assert got["fiber_numbers"] == "7 8 9"
    assert got["states_for_transfer"] == " ".join(str(x) for x in s.states_for_transfer)
    assert got["algebraics_for_transfer"] == "0 4"


@pytest.mark.gpu
@pytest.mark.parametrize("method,precision", [("split", "fp64"), ("fused", "fp32")])
def test_cpp_host_class_equals_python_operator(tmp_path, method, precision):
    exe = _build(tmp_path)
    s = _system()
    cfg = str(tmp_path / "settings.txt")
    S.write_host_settings(s, cfg, method=method, precision=precision)
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, cfg, out, "0.3"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, np.float64)
    ns = 4
    st = raw[:ns * s.n_nodes].reshape(ns, s.n_nodes)
    alg = raw[ns * s.n_nodes:].reshape(2, s.n_nodes)
    with S.FastMonodomainSolver(s.copy(), method=method, precision=precision) as slv:
        slv.setTimeSpan(0.0, 0.3)
        slv.advanceTimeSpan()
        slv.setTimeSpan(0.3, 0.6)
        slv.advanceTimeSpan()
        np.testing.assert_array_equal(st, slv.states())
        np.testing.assert_array_equal(alg, slv.algebraics())
    if precision == "fp64":
        ref, _, _, _ = H.run_oracle(s.copy())
        assert np.max(np.abs(st[0] - ref[0])) <= GP.VM_TOL_FP64


@pytest.mark.gpu
def test_cpp_output_writer_equals_python_writer(tmp_path):
    # the C++ class's writer fires after the same RepeatedCall pieces, with the same names, times and Vm as
    # the Python host class's PythonCallback writer of the same outputInterval
    exe = _build(tmp_path)
    s = _system()
    cfg = str(tmp_path / "settings.txt")
    S.write_host_settings(s, cfg, method="split", precision="fp64")
    out = str(tmp_path / "writes.txt")
    r = subprocess.run([exe, cfg, out, "0", "7"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = [ln.split() for ln in open(out).read().splitlines()]
    got = []
    s2 = s.copy()
    s2.output_writers = [({"format": "PythonCallback", "outputInterval": 7, "filename": "out/fiber",
                           "callback": got.append}, list(range(s.n_fibers)))]
    with S.FastMonodomainSolver(s2, method="split", precision="fp64") as slv:
        slv.advanceTimeSpan()
        slv.callOutputWriter(0, 0.0)
    assert len(lines) == len(got) >= 2
    for (name, t, vm_sum), dicts in zip(lines, got):
        assert float(t) == dicts[0]["currentTime"]
        assert float(vm_sum) == pytest.approx(sum(float(np.sum(d["data"][1]["components"][0]["values"]))
                                                  for d in dicts), rel=1e-13)
    assert lines[0][0] == "out/fiber_0000000"


@pytest.mark.gpu
def test_cpp_stimulation_log_and_equilibrium_equal_python(tmp_path):
    # the C++ class writes the same stimulation log file as the Python host class, and starts from the same
    # equilibrium states when the settings ask for them
    exe = _build(tmp_path)
    s = _system()
    s.end_time = 25.0
    s.fiber_numbers = [4, 5, 6]
    s.initialize_states_to_equilibrium = True
    cfg = str(tmp_path / "settings.txt")
    S.write_host_settings(s, cfg, method="split", precision="fp64")
    out = str(tmp_path / "cpp.log")
    r = subprocess.run([exe, cfg, out, "0", "log"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    s.stimulation_log_filename = str(tmp_path / "py.log")
    slv = S.FastMonodomainSolver(s.copy(), method="split", precision="fp64")
    slv.advanceTimeSpan()
    n = len(slv.stimulation_log()["time"])
    slv.close()
    assert n == 9                          # three fibers stimulated every 10 ms from t = 0
    assert open(out).read() == open(str(tmp_path / "py.log")).read()
    # the default mode writes the states after its advances; with the equilibrium start they equal Python's
    out = str(tmp_path / "out.bin")
    s.end_time = 0.6
    S.write_host_settings(s, cfg, method="split", precision="fp64")
    r = subprocess.run([exe, cfg, out, "0.3"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    st = np.fromfile(out, np.float64)[:4 * s.n_nodes].reshape(4, s.n_nodes)
    with S.FastMonodomainSolver(s.copy(), method="split", precision="fp64") as slv:
        slv.setTimeSpan(0.0, 0.3)
        slv.advanceTimeSpan()
        slv.setTimeSpan(0.3, 0.6)
        slv.advanceTimeSpan()
        np.testing.assert_array_equal(st, slv.states())
        assert slv.equilibrium["max_increment"] < 1e-5
