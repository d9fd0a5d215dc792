"""GPU parity: the CUDA solver (through the C ABI) against the CPU oracle on the same seeded inputs.

Tolerances (from the hot path's specification):
  FP64 paths:            Vm max-abs difference <= 1e-6 mV, activation times equal within one split step;
  FP32-reaction paths:   Vm max-abs difference <= 0.1 mV against the FP64 oracle.
Gating variables are checked at 1e-8 (FP64) / 1e-3 (FP32).
"""
import numpy as np
import pytest

import helpers as H
from opendihu_b200 import solver as S

pytestmark = pytest.mark.gpu

VM_TOL_FP64 = 1e-6
VM_TOL_FP32 = 0.1


def run_gpu(system, method="split", precision="fp64", trace_nodes=(), trace_capacity=0, **kw):
    # "fused" lets the library choose (cluster mode for few fibers); "fused_bins" keeps bins of whole fibers
    if method == "fused_bins":
        method = "fused"
        kw["cluster_size"] = 1
    H.complete(system)
    with S.FastMonodomainSolver(system, method=method, precision=precision, trace_nodes=trace_nodes,
                                trace_capacity=trace_capacity, **kw) as slv:
        slv.setTimeSpan(system.start_time, system.end_time)
        slv.advanceTimeSpan()
        return slv.states(), slv.algebraics(), slv.trace(), slv.split_steps(), slv


def compare(system, method, precision, atol_vm, atol_gates, rtol_states=0.0, **kw):
    ref, ref_alg, _, n_ref = H.run_oracle(system.copy())
    st, alg, _, n, _ = run_gpu(system.copy(), method, precision, **kw)
    assert n == n_ref
    dv = np.max(np.abs(st[0] - ref[0]))
    dg = np.max(np.abs(st[1:] - ref[1:]) - rtol_states * np.abs(ref[1:]))
    assert np.all(np.isfinite(st))
    assert dv <= atol_vm, f"Vm max-abs error {dv}"
    assert dg <= atol_gates, f"gating max-abs error {dg}"
    return st, ref, dv


def small_system(**kw):
    # 3 fibers x 301 nodes (the junction blocks straddle fibers for W=4), stimulated at t = 0
    return H.c1_system(n_fibers=3, n_nodes=301, end_time=kw.pop("end_time", 2.0), **kw)


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins", "auto"])
def test_fp64_matches_oracle(method):
    st, ref, dv = compare(small_system(), method, "fp64", VM_TOL_FP64, 1e-8)
    assert ref[0].max() > 0  # an action potential happened


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins"])
def test_fp32_reaction_within_01mV(method):
    compare(small_system(), method, "fp32", VM_TOL_FP32, 1e-3)


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins"])
def test_crank_nicolson(method):
    compare(small_system(diffusion_scheme="CrankNicolson"), method, "fp64", VM_TOL_FP64, 1e-8)


@pytest.mark.parametrize("method", ["split", "fused"])
def test_approximate_exponential(method):
    compare(small_system(approximate_exponential_function=True), method, "fp64", VM_TOL_FP64, 1e-8)
    compare(small_system(approximate_exponential_function=True), method, "fp32", VM_TOL_FP32, 1e-3)


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins"])
def test_uneven_lengths_center_rule_and_jitter(method):
    rng = np.random.default_rng(3)
    lengths = rng.integers(40, 400, size=7)
    sysm = S.uniform_fibers(H.HH, lengths, 0.01, 3.828 / 500, call_frequency=0.5, repeat_after_first_call=0.1,
                            call_enable_begin=0.05, jitter=rng.uniform(-0.1, 0.1, size=(7, 3)),
                            firing_events=rng.integers(0, 2, size=(5, 4)).astype(np.uint8),
                            motor_unit_no=rng.integers(0, 9, size=7).astype(np.int32), end_time=3.0,
                            clamp_rule="center", diffusion_scheme="CrankNicolson")
    sysm.stimulation_point_index = (lengths * rng.uniform(0.3, 0.7, size=7)).astype(np.int32)
    compare(sysm, method, "fp64", VM_TOL_FP64, 1e-8)


@pytest.mark.parametrize("scheme", ["ImplicitEuler", "CrankNicolson"])
def test_split_many_ragged_fibers(scheme):
    # 200 ragged fibers: the split path's diffusion solves take a CTA per fiber with the fiber staged in shared
    # memory (more fibers than SMs, fewer than the warp-per-fiber threshold)
    rng = np.random.default_rng(11)
    lengths = rng.integers(20, 700, size=200)
    sysm = S.uniform_fibers(H.HH, lengths, 0.01, 3.828 / 500, call_frequency=0.5, repeat_after_first_call=0.1,
                            firing_events=rng.integers(0, 2, size=(4, 6)).astype(np.uint8),
                            motor_unit_no=rng.integers(0, 6, size=200).astype(np.int32), end_time=1.0,
                            clamp_rule="center", diffusion_scheme=scheme)
    compare(sysm, "split", "fp64", VM_TOL_FP64, 1e-8)


@pytest.mark.parametrize("method", ["split", "fused"])
def test_vc_rule_multiple_ranks_and_width8(method):
    compare(small_system(n_ranks=2, vc_width=8), method, "fp64", VM_TOL_FP64, 1e-8)


def test_clamp_nodes_match_oracle():
    sysm = H.c1_system(n_fibers=16, n_nodes=1481, end_time=0.0)
    H.complete(sysm)
    with S.FastMonodomainSolver(sysm) as slv:
        first, cnt, ev = slv.clamp_nodes()
    run = H.O.OracleRun(H.oracle_spec(sysm))
    of, oc = run.vc_clamp_nodes()
    np.testing.assert_array_equal(first, of)
    np.testing.assert_array_equal(cnt, oc)
    assert first[0] == 740 and first[1] == 1481 + 739  # the W=4 buffer rule shifts the clamp per fiber


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins"])
def test_current_stimulus_mode(method):
    # the benchmark's 1200 uA/cm^2 current at the junction for 0.1 ms every 10 ms (parameter 0 = I_Stim)
    sysm = small_system(stimulus_mode="current", stimulus_parameter=0, stimulus_value=1200.0)
    st, ref, dv = compare(sysm, method, "fp64", VM_TOL_FP64, 1e-8)
    assert ref[0].max() > 0


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins"])
def test_per_node_parameters_and_prefactor(method):
    sysm = small_system()
    H.complete(sysm)
    rng = np.random.default_rng(5)
    sysm.prefactor = rng.uniform(2.5, 5.0, size=sysm.n_fibers) / 500.0
    scale = np.repeat(rng.uniform(0.8, 1.2, size=(2, sysm.n_fibers)), np.diff(sysm.fiber_offsets), axis=1)
    sysm.parameters[1] *= scale[0]
    sysm.parameters[2] *= scale[1]
    compare(sysm, method, "fp64", VM_TOL_FP64, 1e-8)


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins"])
def test_algebraics_for_transfer(method):
    sysm = small_system(end_time=0.5, algebraics_for_transfer=[0, 4, 8])
    ref, ref_alg, _, _ = H.run_oracle(sysm.copy())
    st, alg, _, _, _ = run_gpu(sysm.copy(), method)
    np.testing.assert_allclose(alg, ref_alg, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins"])
def test_repeated_advances_and_checkpoint(method):
    sysm = small_system(end_time=1.0)
    H.complete(sysm)
    kw = {"method": "fused", "cluster_size": 1} if method == "fused_bins" else {"method": method}
    with S.FastMonodomainSolver(sysm, steps_per_launch=37, **kw) as slv:
        slv.setTimeSpan(0.0, 0.4)
        slv.advanceTimeSpan()
        slv.saveFiberDataCheckpoint()
        slv.setTimeSpan(0.4, 1.0)
        slv.advanceTimeSpan()
        a = slv.states()
        slv.restoreFiberDataCheckpoint()
        slv.setTimeSpan(0.4, 1.0)
        slv.advanceTimeSpan()
        b = slv.states()
    np.testing.assert_array_equal(a, b)
    # two advances == the oracle run over the whole span (the stimulation machine state carries over)
    spec = H.oracle_spec(sysm.copy())
    run = H.O.OracleRun(spec)
    st = sysm.states.copy()
    run.run(st, 0.0, 0.4)
    run.run(st, 0.4, 1.0)
    assert np.max(np.abs(a[0] - st[0])) <= VM_TOL_FP64


@pytest.mark.parametrize("method", ["split", "fused", "fused_bins"])
def test_window_sizes_do_not_change_results(method):
    sysm = small_system(end_time=0.7)
    H.complete(sysm)
    outs = []
    for k in (1, 7, 100):
        st, _, _, _, _ = run_gpu(sysm.copy(), method, steps_per_launch=k)
        outs.append(st)
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])


@pytest.mark.parametrize("shape", [(128, 8), (256, 4), (512, 3), (1024, 3)])
def test_fused_shapes_agree(shape):
    sysm = H.c1_system(n_fibers=4, n_nodes=257, end_time=0.5)
    H.complete(sysm)
    ref, _, _, _ = H.run_oracle(sysm.copy())
    st, _, _, _, _ = run_gpu(sysm.copy(), "fused", threads_per_block=shape[0], nodes_per_thread=shape[1])
    assert np.max(np.abs(st[0] - ref[0])) <= VM_TOL_FP64


def test_shorten_split_fp64_and_fp32():
    sysm = S.uniform_fibers(H.SHORTEN, [61, 47], 0.01, 3.828 / (500 * 0.58), call_frequency=0.1,
                            repeat_after_first_call=0.1, end_time=0.05, dt_0d=1e-5, dt_1d=5e-4, dt_splitting=5e-4,
                            dt_repeated_call=5e-4)
    compare(sysm.copy(), "split", "fp64", VM_TOL_FP64, 1e-6)
    # Shorten's states span 1e-6 .. 2e4 (concentrations): relative tolerance for the FP32 states
    compare(sysm.copy(), "split", "fp32", VM_TOL_FP32, 1e-4, rtol_states=1e-3)


def test_nan_is_reported():
    sysm = small_system(end_time=0.01)
    H.complete(sysm)
    sysm.states[0, 5] = np.nan
    with pytest.raises(S.N.FdmError) as e:
        run_gpu(sysm, "split")
    assert e.value.code == S.N.FDM_ERR_NAN


@pytest.mark.slow
@pytest.mark.parametrize("method,precision", [("split", "fp64"), ("fused", "fp64"), ("fused", "fp32"),
                                              ("fused_bins", "fp64")])
def test_plain_method_config_10ms(method, precision):
    """16 HH fibers x 1481 nodes, 10 ms: Vm after 10 ms and activation times against the oracle."""
    sysm = H.c1_system(end_time=10.0)
    H.complete(sysm)
    nodes = [f * 1481 + k for f in (0, 7, 15) for k in (740, 800, 900, 1000, 1480)]
    ref, _, tr_ref, n = H.run_oracle(sysm.copy(), trace_nodes=nodes, trace_capacity=10000)
    st, _, tr, n2, _ = run_gpu(sysm.copy(), method, precision, trace_nodes=nodes, trace_capacity=10000)
    assert n == n2 == 10000
    tol = VM_TOL_FP64 if precision == "fp64" else VM_TOL_FP32
    assert np.max(np.abs(st[0] - ref[0])) <= tol
    at_ref = H.activation_times(tr_ref, 1e-3)
    at = H.activation_times(tr, 1e-3)
    assert np.array_equal(np.isnan(at), np.isnan(at_ref))
    ok = ~np.isnan(at)
    assert np.all(np.abs(at[ok] - at_ref[ok]) <= 1e-3 + 1e-12)


def test_asynchronous_advance_equals_blocking():
    sysm = small_system(end_time=0.6)
    H.complete(sysm)
    with S.FastMonodomainSolver(sysm.copy(), method="fused") as a, S.FastMonodomainSolver(sysm.copy(), method="fused") as b:
        a.setTimeSpan(0.0, 0.3)
        a.advanceTimeSpan()
        a.setTimeSpan(0.3, 0.6)
        a.advanceTimeSpan()
        b.setTimeSpan(0.0, 0.3)
        b.advance_async()
        b.setTimeSpan(0.3, 0.6)
        b.advance_async()            # waits for the first one itself
        b.wait()
        np.testing.assert_array_equal(a.states(), b.states())
        assert b.timing()["advance_ms"] > 0
    bad = small_system(end_time=0.01)
    H.complete(bad)
    bad.states[0, 5] = np.nan
    with S.FastMonodomainSolver(bad, method="split") as c:
        c.advance_async()
        with pytest.raises(S.N.FdmError) as e:
            c.wait()
        assert e.value.code == S.N.FDM_ERR_NAN
