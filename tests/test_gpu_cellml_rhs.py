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
