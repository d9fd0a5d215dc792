"""A run-time model module on the GPU: the HH variant with g_Na and g_L as parameters (g_K and i_Stim constants),
generated, compiled and loaded at run time, against the oracle's built-in HH (the same equations with g_L and
g_K at their constant values): split FP64 to 1e-6 mV, FP32 reaction to 0.1 mV, the equilibrium skip, the adjoint
against the built-in model's adjoint, and the fused method refused (modules carry the split-path kernels)."""
import numpy as np
import pytest

import helpers as H
from opendihu_b200 import _native as N
from opendihu_b200 import models as MD
from opendihu_b200 import solver as S

pytestmark = pytest.mark.gpu

VARIANT = ((), (3, 5))


def _systems(end_time=2.0, **kw):
    name = MD.load_model(H.HH, *VARIANT)
    base = H.c1_system(n_fibers=3, n_nodes=201, end_time=end_time, **kw)
    H.complete(base)
    g_na = np.repeat(np.array([100.0, 120.0, 140.0]), 201)
    base.parameters[1] = g_na                       # built-in slots: i_Stim, g_Na, g_K
    mod = base.copy()
    mod.model = name
    mod.parameters = np.stack([g_na, np.full(base.n_nodes, 0.3)])   # module slots: g_Na, g_L
    return base, mod


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("fp32", 0.1)])
def test_module_matches_oracle(precision, tol):
    base, mod = _systems()
    ref, _, _, n = H.run_oracle(base.copy())
    with S.FastMonodomainSolver(mod.copy(), method="split", precision=precision) as slv:
        slv.advanceTimeSpan()
        st = slv.states()
        assert slv.split_steps() == n
    assert ref[0].max() > 0                         # an action potential
    assert np.max(np.abs(st[0] - ref[0])) <= tol


def test_module_equilibrium_skip_matches_oracle():
    base, mod = _systems(end_time=3.0)
    base.skip_close_to_equilibrium = mod.skip_close_to_equilibrium = True
    ref, _, _, _ = H.run_oracle(base.copy())
    with S.FastMonodomainSolver(mod.copy(), method="split", precision="fp64") as slv:
        slv.advanceTimeSpan()
        st = slv.states()
    assert np.max(np.abs(st[0] - ref[0])) <= 1e-6


def test_module_adjoint_equals_builtin_adjoint():
    from opendihu_b200 import adjoint as ADJ
    base, mod = _systems(end_time=0.3)
    sensors = np.array([0, 100, 200, 250, 500])
    out = {}
    for key, sysm in (("builtin", base), ("module", mod)):
        eng = ADJ.AdjointEngine(sysm, sensors, checkpoint_every=40)
        try:
            tr = eng.forward(sysm.prefactor, sysm.parameters)
            g = eng.backward(np.ones_like(tr))
        finally:
            eng.close()
        out[key] = (tr, g)
    np.testing.assert_allclose(out["module"][0], out["builtin"][0], rtol=0, atol=1e-9)
    np.testing.assert_allclose(out["module"][1]["prefactor"], out["builtin"][1]["prefactor"], rtol=1e-8)
    # dL/dg_Na: module slot 0, built-in slot 1
    np.testing.assert_allclose(out["module"][1]["parameters"][0], out["builtin"][1]["parameters"][1], rtol=1e-8,
                               atol=1e-12 * np.abs(out["builtin"][1]["parameters"][1]).max())


def test_module_rhs_device_function_matches_oracle():
    import ctypes as C
    import torch
    from oracle import oracle as O
    name = MD.load_model(H.HH, *VARIANT)
    n = 64
    rng = np.random.default_rng(5)
    states = np.stack([rng.uniform(-80, 30, n), rng.uniform(0, 1, n), rng.uniform(0, 1, n), rng.uniform(0, 1, n)])
    g_na = rng.uniform(100, 140, n)
    dev = torch.device("cuda:0")
    st_d = torch.from_numpy(states.copy()).to(dev)
    p_d = torch.from_numpy(np.stack([g_na, np.full(n, 0.3)])).to(dev)
    r_d = torch.zeros_like(st_d)
    N.check(N.lib().fdm_cellml_rhs_device(N.MODEL_IDS[name], 0, n, 0.0, C.c_void_p(st_d.data_ptr()),
                                          C.c_void_p(p_d.data_ptr()), C.c_void_p(r_d.data_ptr()), None, None))
    torch.cuda.synchronize()
    got = r_d.cpu().numpy()
    for i in range(n):
        r = O.rates(H.HH, states[:, i], np.array([0.0, g_na[i], 36.0]))[0]
        np.testing.assert_allclose(got[:, i], r, rtol=1e-12, atol=1e-12)


def test_fused_method_is_refused_for_a_module_and_auto_picks_split():
    base, mod = _systems(end_time=0.05)
    with pytest.raises(N.FdmError) as e:
        with S.FastMonodomainSolver(mod.copy(), method="fused", precision="fp32") as slv:
            slv.advanceTimeSpan()
    assert e.value.code == N.FDM_ERR_UNSUPPORTED
    with S.FastMonodomainSolver(mod.copy(), method="auto", precision="fp32") as slv:
        slv.advanceTimeSpan()
        assert slv.method == "split"
