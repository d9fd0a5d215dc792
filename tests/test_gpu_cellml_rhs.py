"""The CellmlAdapter's generic right-hand side (the non-fast path's computeCellMLRightHandSide) on the GPU:
device-pointer entry and the reference-signature export, against the oracle's right-hand side."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from oracle import oracle as O
from opendihu_b200 import _native as N

pytestmark = pytest.mark.gpu


def _inputs(model, n, seed):
    rng = np.random.default_rng(seed)
    ns, na, npar, init = O.model_info(model)
    states = init[:, None] * (1 + 0.05 * rng.standard_normal((ns, n)))
    params = H.default_parameters(model, n) * (1 + 0.1 * rng.standard_normal((npar, n)))
    return states, params, ns, na


def _oracle(model, states, params, t, approx):
    ns = states.shape[0]
    r = np.zeros_like(states)
    algs = []
    for i in range(states.shape[1]):
        ri, ai = O.rates(model, states[:, i], params[:, i], t, approx)
        r[:, i] = ri[:ns]
        algs.append(ai)
    return r, np.array(algs).T


@pytest.mark.parametrize("model,approx", [(H.HH, False), (H.HH, True), (H.SHORTEN, False)])
def test_device_entry_matches_oracle(model, approx):
    torch = pytest.importorskip("torch")
    n = 1000
    states, params, ns, na = _inputs(model, n, 1)
    ref_r, ref_a = _oracle(model, states, params, 0.25, approx)
    dev = torch.device("cuda:0")
    st = torch.tensor(states, dtype=torch.float64, device=dev).contiguous()
    pr = torch.tensor(params, dtype=torch.float64, device=dev).contiguous()
    r = torch.zeros((ns, n), dtype=torch.float64, device=dev)
    a = torch.zeros((na, n), dtype=torch.float64, device=dev)
    N.check(N.lib().fdm_cellml_rhs_device(N.MODEL_IDS[model], int(approx), n, 0.25, C.c_void_p(st.data_ptr()),
                                          C.c_void_p(pr.data_ptr()), C.c_void_p(r.data_ptr()),
                                          C.c_void_p(a.data_ptr()), None))
    torch.cuda.synchronize()
    np.testing.assert_allclose(r.cpu().numpy(), ref_r, rtol=1e-11, atol=1e-12 * np.abs(ref_r).max())
    np.testing.assert_allclose(a.cpu().numpy(), ref_a[:na], rtol=1e-11, atol=1e-12 * np.abs(ref_a).max())


def test_reference_signature_export():
    n = 777
    states, params, ns, na = _inputs(H.HH, n, 2)
    ref_r, ref_a = _oracle(H.HH, states, params, 0.0, False)
    L = N.lib()
    N.check(L.fdm_cellml_rhs_configure(N.MODEL_IDS[H.HH], n, 0, 0))
    st = np.ascontiguousarray(states)
    pr = np.ascontiguousarray(params)
    r = np.zeros((ns, n))
    a = np.zeros((na, n))
    L.computeCellMLRightHandSide(None, 0.0, N.ptr(st, C.c_double), N.ptr(r, C.c_double), N.ptr(a, C.c_double),
                                 N.ptr(pr, C.c_double))
    np.testing.assert_allclose(r, ref_r, rtol=1e-11, atol=1e-12 * np.abs(ref_r).max())
    np.testing.assert_allclose(a, ref_a[:na], rtol=1e-11, atol=1e-12 * np.abs(ref_a).max())


def _rk4_increment(y, P, dt, approx=False):
    f = lambda u, t: O.rates(H.HH, u, P, t, approx=approx)[0]
    k1 = f(y, 0.0)
    k2 = f(y + dt / 2. * k1, dt / 2.)
    k3 = f(y + dt / 2. * k2, dt / 2.)
    k4 = f(y + dt * k3, dt)
    return (k1 + 2 * k2 + 2 * k3 + k4) / 6.


def test_equilibrium_search():
    # initializeStatesToEquilibrium (03_cellml_adapter.tpp:445-515) for HH from its initial values: the same RK4
    # search with the oracle's right-hand side on the CPU stops after 436,094 steps at the values below
    from opendihu_b200 import solver as S
    s = H.complete(H.c1_system(n_fibers=1, n_nodes=3, end_time=0.0))
    eq = S.equilibrium_states(s)
    assert eq["max_increment"] < 1e-5 and eq["dt"] == 1e-4
    assert 436_000 <= eq["iterations"] <= 436_200
    np.testing.assert_allclose(eq["states"], [-7.49951664e+01, 5.29626812e-02, 5.96036857e-01, 3.17728799e-01],
                               rtol=1e-6)
    assert np.max(np.abs(_rk4_increment(eq["states"], s.parameters[:, 0], 1e-4))) < 1.001e-5


def test_settings_initialize_states_to_equilibrium():
    from test_only_if_stimulated import reference_settings
    from opendihu_b200 import solver as S
    cfg = reference_settings(n_fibers=2)
    for inst in cfg["RepeatedCall"]["MultipleInstances"]["instances"][0]["StrangSplitting"]["Term1"][
            "MultipleInstances"]["instances"]:
        inst["Heun"]["CellML"]["initializeStatesToEquilibrium"] = True
        inst["Heun"]["CellML"]["initializeStatesToEquilibriumTimestepWidth"] = 2e-4
    s = S.parse_settings(cfg)
    assert s.initialize_states_to_equilibrium and s.equilibrium_dt == 2e-4
    assert s.approximate_exponential_function       # the vc default: the search uses the approximate exp too
    with S.FastMonodomainSolver(s, method="split", precision="fp64") as slv:
        st = slv.states()
        eq = slv.equilibrium["states"]
    np.testing.assert_array_equal(st, np.repeat(eq[:, None], st.shape[1], axis=1))
    assert np.max(np.abs(_rk4_increment(eq, s.parameters[:, 0], 2e-4, approx=True))) < 1.001e-5
