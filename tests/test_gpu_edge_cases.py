"""Edge cases against the oracle: the smallest fibers (2 nodes), many short fibers (more than the 32 fibers a
fused bin holds), junctions at the first and the last node, W = 1, firing tables and jitter lists that wrap,
a span shorter than one split step, no fibers at all, and a fiber longer than every fused bin."""
import numpy as np
import pytest

import helpers as H
import test_gpu_parity as GP
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", ["split", "fused"])
def test_two_node_fibers_and_many_short_fibers(method):
    rng = np.random.default_rng(11)
    lengths = np.concatenate([[2, 2, 3], rng.integers(2, 12, size=70)])
    s = S.uniform_fibers(H.HH, lengths, 0.01, 3.828 / 500, call_frequency=0.2, repeat_after_first_call=0.1,
                         firing_events=rng.integers(0, 2, size=(7, 3)).astype(np.uint8),
                         motor_unit_no=rng.integers(0, 10, size=len(lengths)).astype(np.int32), end_time=1.5)
    GP.compare(s, method, "fp64", GP.VM_TOL_FP64, 1e-8)


@pytest.mark.parametrize("method,rule", [("split", "vc"), ("fused", "vc"), ("split", "center"), ("fused", "center")])
def test_junction_at_the_fiber_ends(method, rule):
    s = WL.batched_hh(n_fibers=6, min_nodes=20, max_nodes=45, seed=12, end_time=1.0, clamp_rule=rule)
    lengths = np.diff(s.fiber_offsets)
    s.stimulation_point_index = np.where(np.arange(6) % 2 == 0, 0, lengths - 1).astype(np.int32)
    GP.compare(s, method, "fp64", GP.VM_TOL_FP64, 1e-8)


@pytest.mark.parametrize("method", ["split", "fused"])
def test_lane_width_one_and_wrapping_tables(method):
    rng = np.random.default_rng(13)
    s = WL.batched_hh(clamp_rule="vc", n_fibers=5, min_nodes=30, max_nodes=50, seed=13, end_time=2.0, vc_width=1, n_ranks=2)
    s.firing_events = rng.integers(0, 2, size=(3, 2)).astype(np.uint8)      # rows and motor units wrap
    s.motor_unit_no = np.array([0, 1, 5, 8, 13], np.int32)
    s.call_frequency = np.full(5, 2.0)
    s.jitter = rng.uniform(-0.3, 0.3, size=(5, 2))                           # jitter index wraps
    GP.compare(s, method, "fp64", GP.VM_TOL_FP64, 1e-8)


@pytest.mark.parametrize("method", ["split", "fused"])
def test_span_shorter_than_a_split_step(method):
    s = GP.small_system(end_time=0.0004)
    ref, _, _, n = H.run_oracle(s.copy())
    st, _, _, n2, _ = GP.run_gpu(s.copy(), method)
    assert n == n2 == 1
    assert np.max(np.abs(st[0] - ref[0])) <= GP.VM_TOL_FP64


def test_no_fibers():
    s = S.uniform_fibers(H.HH, [], 0.01, 3.828 / 500, end_time=0.2)
    s.states = np.zeros((4, 0))
    s.parameters = np.zeros((3, 0))
    with S.FastMonodomainSolver(s, method="split") as slv:
        slv.advanceTimeSpan()
        assert slv.states().shape == (4, 0)


def test_fiber_longer_than_every_fused_launch_fails_loudly():
    longest = max(t * m for t, m in S.N.fused_shapes())
    s = S.uniform_fibers(H.HH, [longest + 1], 0.01, 3.828 / 500, end_time=0.01)
    with pytest.raises(S.N.FdmError) as e:
        S.FastMonodomainSolver(H.complete(s.copy()), method="fused", cluster_size=1).initialize()
    assert e.value.code == S.N.FDM_ERR_UNSUPPORTED
    # cluster mode holds up to 8 CTAs of its largest shape per fiber
    longest_cluster = 8 * max(t * m for t, m in S.N.fused_shapes(cluster=True))
    s = S.uniform_fibers(H.HH, [longest_cluster + 1], 0.01, 3.828 / 500, end_time=0.01)
    with pytest.raises(S.N.FdmError) as e:
        S.FastMonodomainSolver(H.complete(s), method="fused").initialize()
    assert e.value.code == S.N.FDM_ERR_UNSUPPORTED


@pytest.mark.parametrize("n_fibers", [591, 592])
def test_split_diffusion_on_both_sides_of_the_block_threshold(n_fibers):
    # below 592 fibers the split path solves each fiber with a CTA, from 592 on with a warp
    rng = np.random.default_rng(n_fibers)
    lengths = rng.integers(2, 40, size=n_fibers)
    s = S.uniform_fibers(H.HH, lengths, 0.01, 3.828 / 500, call_frequency=0.2, repeat_after_first_call=0.1,
                         firing_events=rng.integers(0, 2, size=(5, 4)).astype(np.uint8),
                         motor_unit_no=rng.integers(0, 4, size=n_fibers).astype(np.int32), end_time=0.6,
                         diffusion_scheme="CrankNicolson")
    GP.compare(s, "split", "fp64", GP.VM_TOL_FP64, 1e-8)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_page_locked_state_arrays_transfer_like_pageable_ones(precision):
    # fdm_host_alloc memory is moved by DMA directly (FP32 mode: converted on the device); pageable arrays go
    # through the staging copy: the same bits either way, in both directions
    from opendihu_b200 import _native as N
    s = WL.batched_hh(n_fibers=40, seed=5, end_time=0.5)
    H.complete(s)
    with S.FastMonodomainSolver(s.copy(), method="fused", precision=precision) as slv:
        slv.advanceTimeSpan()
        pageable = slv.states()
        pinned = slv.states(out=slv.pinned_states())
        assert np.array_equal(pageable.view(np.int64), pinned.view(np.int64))
        rng = np.random.default_rng(1)
        new = pageable + rng.normal(scale=1e-3, size=pageable.shape)
        src = slv.pinned_states()
        src[...] = new
        slv.set_states(src)
        a = slv.states()
        slv.set_states(new)
        b = slv.states(out=slv.pinned_states())
        assert np.array_equal(a.view(np.int64), b.view(np.int64))
        if precision == "fp64":
            assert np.array_equal(a.view(np.int64), new.view(np.int64))
        else:
            # FP32 mode keeps (value, residual) pairs: FP64 values survive the round trip to ~1e-14 relative
            np.testing.assert_allclose(a, new, rtol=1e-13, atol=1e-300)
    buf = np.zeros(4)
    import ctypes as C
    assert N.lib().fdm_host_free(buf.ctypes.data_as(C.c_void_p)) == N.FDM_ERR_ARG
