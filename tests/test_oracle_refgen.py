"""The oracle's Heun step against the reference's own generated code (no GPU).

oracle/Makefile (target ref, where the reference checkout exists) compiles the reference's CellML code
generator from its sources and builds the FastMonodomainSolver code it emits: compute0DInstance, one Heun step
of a W = 4 lane point buffer with the clamp of lanes 0..2 and the algebraics-for-transfer store
(03_generator_vc.cpp:873-1163).  The oracle's restatement (oracle_heun_buffer, fdm_oracle.c heun_step) must
give the same states and algebraics, bit for bit, over hundreds of steps, with and without the clamp, for
both models and both exponential variants.
"""
import ctypes as C
import os

import numpy as np
import pytest

import helpers as H
from oracle import oracle as O

REF_DIR = os.path.join(H.ROOT, "oracle", "_ref")
ORACLE = os.path.join(H.ROOT, "oracle", "liboracle.so")

CASES = [  # (library, model, approximate exponential, dt, transferred algebraics)
    ("libref_hh_fast_approx.so", H.HH, 1, 1e-4, [0, 4, 8]),
    ("libref_hh_fast_exact.so", H.HH, 0, 1e-4, [0, 4, 8]),
    ("libref_shorten_fast_exact.so", H.SHORTEN, 0, 1e-5, [0, 4, 10, 31]),
]


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _libs(name):
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (make -C oracle ref needs the reference checkout)")
    R = C.CDLL(path)
    R.refgen_heun_buffer.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                     C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_double)]
    L = C.CDLL(ORACLE)
    L.oracle_heun_buffer.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int,
                                     C.POINTER(C.c_int), C.POINTER(C.c_double)]
    return R, L


@pytest.mark.parametrize("stimulate", [0, 1], ids=["free", "clamped"])
@pytest.mark.parametrize("lib,model,approx,dt,alg", CASES, ids=["hh_approx", "hh_exact", "shorten_exact"])
def test_oracle_heun_equals_reference_generated_code(lib, model, approx, dt, alg, stimulate):
    R, L = _libs(lib)
    W = R.refgen_lanes()
    assert W == 4
    ns, na, npar, init = O.model_info(model)
    # four lanes at different points of an action potential; per-lane parameters
    y0 = np.repeat(init[:, None], W, axis=1)
    y0[0] = init[0] + np.array([0.0, 15.0, 55.0, 85.0])
    params = np.repeat((np.array([0.0, 120.0, 36.0]) if model == H.HH else np.array([0.0, 1.0]))[:, None], W, axis=1)
    params = params * np.array([1.0, 0.9, 1.1, 1.05])[None, :]
    idx = np.array(alg, np.int32)
    mid = O.MODELS[model]
    for t0, n_steps in ((0.0, 1), (0.35, 300)):
        a = y0.ravel().copy()
        b = a.copy()
        pa = np.ascontiguousarray(params.ravel())
        alg_a = np.zeros(len(idx) * W)
        alg_b = np.zeros(len(idx) * W)
        R.refgen_heun_buffer(ns, npar, _p(a, C.c_double), _p(pa, C.c_double), t0, dt, n_steps, stimulate, 20.0,
                             len(idx), _p(idx, C.c_int), _p(alg_a, C.c_double))
        assert L.oracle_heun_buffer(mid, W, approx, _p(b, C.c_double), _p(pa, C.c_double), t0, dt, n_steps,
                                    stimulate, 20.0, len(idx), _p(idx, C.c_int), _p(alg_b, C.c_double)) == 0
        assert np.max(np.abs(a - y0.ravel())) > 0                 # the states moved
        np.testing.assert_array_equal(a, b)                          # bit for bit
        np.testing.assert_array_equal(alg_a, alg_b)
        if stimulate:
            np.testing.assert_array_equal(a[:3], 20.0)               # lanes 0..2 clamped, lane 3 free
            assert a[3] != 20.0
