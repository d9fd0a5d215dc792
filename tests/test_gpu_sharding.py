"""Sharded solves on the GPU: an LPT-sharded system (three shards on one device, concurrent host threads and
streams) reproduces the unsharded solve, under the layout-dependent "vc" clamp rule too, and its adjoint
gradients equal the unsharded adjoint's."""
import numpy as np
import pytest

import helpers as H
from opendihu_b200 import sharding as SH
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def _system(**kw):
    kw.setdefault("clamp_rule", "vc")
    s = WL.batched_hh(n_fibers=37, min_nodes=60, max_nodes=400, seed=11, end_time=kw.pop("end_time", 3.0), **kw)
    s.call_enable_begin[:] = 0.0
    return H.complete(s)


def _unsharded(system, **kw):
    with S.FastMonodomainSolver(system.copy(), **kw) as slv:
        slv.advanceTimeSpan()
        return slv.states()


@pytest.mark.parametrize("method,n_ranks", [("split", 1), ("split", 2), ("fused", 1)])
def test_sharded_equals_unsharded(method, n_ranks):
    s = _system(n_ranks=n_ranks)
    ref = _unsharded(s, method=method)
    sh = SH.ShardedSolver(s.copy(), devices=[0], n_shards=3, method=method)
    with sh:
        sh.advanceTimeSpan()
        st = sh.states()
        first, cnt, _ = SH.global_clamp_nodes(s)
        for k, sv in enumerate(sh.shards):
            lf, lc, _ = sv.clamp_nodes()
            np.testing.assert_array_equal(lc, cnt[sh.fibers[k]])
    if method == "split":
        np.testing.assert_array_equal(st, ref)     # same kernels, every fiber independent of its neighbours
    else:
        assert np.max(np.abs(st[0] - ref[0])) <= 1e-9   # the block scan's tree depends on the bin layout
    assert np.max(np.abs(st[0] - H.run_oracle(s.copy())[0][0])) <= 1e-6


def test_sharded_adjoint_equals_unsharded():
    s = _system(end_time=1.0)
    sensors = np.asarray(s.fiber_offsets[:-1]) + 30
    with S.FastMonodomainSolver(s.copy()) as slv:
        tr = slv.adjoint_forward(s.start_time, s.end_time, 50, sensors)
        g = slv.adjoint_backward(np.ones_like(tr))
    with SH.ShardedSolver(s.copy(), devices=[0], n_shards=2) as sh:
        tr2 = sh.adjoint_forward(s.start_time, s.end_time, 50, sensors)
        g2 = sh.adjoint_backward(np.ones_like(tr2))
    np.testing.assert_array_equal(tr2, tr)
    for k in ("prefactor", "parameters", "states0"):
        np.testing.assert_allclose(g2[k], g[k], rtol=1e-12, atol=1e-300)


def test_sharded_only_if_stimulated_equals_unsharded():
    s = _system(clamp_rule="center")
    s.only_compute_if_has_been_stimulated = True
    s.call_enable_begin = np.linspace(0.0, 2.0, s.n_fibers)
    ref = _unsharded(s)
    with SH.ShardedSolver(s.copy(), devices=[0], n_shards=3) as sh:
        sh.advanceTimeSpan()
        st = sh.states()
    np.testing.assert_array_equal(st, ref)


def test_sequential_shard_adjoint_equals_unsharded():
    s = _system(end_time=1.0)
    sensors = np.asarray(s.fiber_offsets[:-1]) + 30
    rng = np.random.default_rng(12)
    with S.FastMonodomainSolver(s.copy()) as slv:
        tr = slv.adjoint_forward(s.start_time, s.end_time, 50, sensors)
        w = rng.standard_normal(tr.shape)
        g = slv.adjoint_backward(w)
    per_node = SH.plan_adjoint(s, s.start_time, s.end_time, 1e15)["bytes_per_node"]
    plan = SH.plan_adjoint(s, s.start_time, s.end_time, s.n_nodes * per_node / 2.5)
    assert plan["n_shards"] >= 3
    with SH.ShardedSolver(s.copy(), devices=[0], n_shards=plan["n_shards"]) as sh:
        tr2, g2 = sh.adjoint(s.start_time, s.end_time, plan["checkpoint_every"], sensors,
                             lambda trace, cols: w[:trace.shape[0], cols])
    np.testing.assert_array_equal(tr2, tr)
    for k in ("prefactor", "parameters", "states0"):
        np.testing.assert_allclose(g2[k], g[k], rtol=1e-12, atol=1e-300)
