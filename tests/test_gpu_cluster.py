"""Cluster mode of the fused kernel (a fiber spread over the CTAs of one thread-block cluster, the tridiagonal
scan carried across them through distributed shared memory) against the oracle: chosen automatically for
few fibers and for fibers longer than every bin, forced cluster sizes 2..8 on ragged fibers (CTAs past a
fiber's end included), Crank-Nicolson, FP32 reaction, traces and algebraicsForTransfer, and its agreement
with the bins of whole fibers."""
import numpy as np
import pytest

import helpers as H
import test_gpu_parity as GP
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def _layout(system, **kw):
    with S.FastMonodomainSolver(H.complete(system.copy()), method="fused", **kw) as slv:
        slv.initialize()
        return slv.fused_layout()


def test_few_fibers_choose_cluster_mode_and_match_oracle():
    s = H.c1_system(n_fibers=16, n_nodes=1481, end_time=0.6)
    lay = _layout(s)
    assert lay["cluster_size"] > 1 and lay["n_blocks"] == 16 * lay["cluster_size"]
    assert _layout(s, cluster_size=1)["cluster_size"] == 1
    st, ref, dv = GP.compare(s, "fused", "fp64", GP.VM_TOL_FP64, 1e-8)
    assert ref[0].max() > 0
    bins, _, _, _, _ = GP.run_gpu(s.copy(), "fused_bins")
    assert np.max(np.abs(st - bins)) <= 1e-9   # only the scan's tree differs


def test_many_fibers_keep_bins():
    s = WL.batched_hh(clamp_rule="vc", n_fibers=600, min_nodes=500, max_nodes=900, seed=1, end_time=0.0)
    assert _layout(s)["cluster_size"] == 1


@pytest.mark.parametrize("csize", [2, 3, 5, 8])
def test_forced_cluster_sizes_ragged_fibers(csize):
    rng = np.random.default_rng(csize)
    cap = 128 * 2
    lengths = np.concatenate([[2, cap * csize, cap * (csize - 1) + 1], rng.integers(3, cap * csize, size=6)])
    s = S.uniform_fibers(H.HH, lengths, 0.01, 3.828 / 500, call_frequency=0.2, repeat_after_first_call=0.1,
                         end_time=0.8, diffusion_scheme="CrankNicolson")
    s.stimulation_point_index = rng.integers(0, lengths).astype(np.int32)
    kw = dict(cluster_size=csize, threads_per_block=128, nodes_per_thread=2)
    lay = _layout(s, **kw)
    assert (lay["threads"], lay["nodes_per_thread"], lay["cluster_size"]) == (128, 2, csize)
    GP.compare(s, "fused", "fp64", GP.VM_TOL_FP64, 1e-8, **kw)


@pytest.mark.parametrize("shape", [(128, 2), (256, 2), (512, 2), (256, 4), (192, 1), (256, 1)])
def test_cluster_shapes_fp32_within_01mV(shape):
    s = H.c1_system(n_fibers=5, n_nodes=1481, end_time=1.0)
    kw = dict(threads_per_block=shape[0], nodes_per_thread=shape[1], cluster_size=-(-1481 // (shape[0] * shape[1])))
    GP.compare(s, "fused", "fp32", GP.VM_TOL_FP32, 1e-3, **kw)


def test_traces_and_algebraics_in_cluster_mode():
    s = H.c1_system(n_fibers=3, n_nodes=1481, end_time=0.5, algebraics_for_transfer=[0, 4, 8])
    H.complete(s)
    nodes = [f * 1481 + k for f in range(3) for k in (0, 255, 256, 740, 1023, 1024, 1480)]
    ref, ref_alg, tr_ref, n = H.run_oracle(s.copy(), trace_nodes=nodes, trace_capacity=1000)
    st, alg, tr, n2, slv = GP.run_gpu(s.copy(), "fused", trace_nodes=nodes, trace_capacity=1000)
    assert n == n2 == 500
    np.testing.assert_allclose(tr, tr_ref, rtol=0, atol=GP.VM_TOL_FP64)
    np.testing.assert_allclose(alg, ref_alg, rtol=1e-9, atol=1e-9)


def test_fiber_longer_than_every_bin_runs_in_cluster_mode():
    longest = max(t * m for t, m in S.N.fused_shapes())
    s = S.uniform_fibers(H.HH, [longest + 1, 700], 0.01, 3.828 / 500, end_time=0.3)
    lay = _layout(s)
    assert lay["cluster_size"] > 1
    GP.compare(s, "fused", "fp64", GP.VM_TOL_FP64, 1e-8)


def test_autotuner_considers_cluster_shapes():
    from opendihu_b200 import autotune as AT
    s = H.complete(H.c1_system(n_fibers=4, n_nodes=1481, end_time=0.3))
    res = AT.autotune(s, "fp64", n_steps=5, steps_per_launch=(50,), use_cache=False)
    assert any(t.get("cluster_size", 1) > 1 for t in res["trials"])
    assert any(t.get("cluster_size", 1) == 1 for t in res["trials"])
    with S.FastMonodomainSolver(s.copy(), method="fused", precision="fp64", autotune=True) as slv:
        slv.advanceTimeSpan()
        lay = slv.fused_layout()
        st = slv.states()
    assert lay["cluster_size"] == slv.tuning["cluster_size"]
    ref, _, _, _ = H.run_oracle(s.copy())
    assert np.max(np.abs(st[0] - ref[0])) <= GP.VM_TOL_FP64
