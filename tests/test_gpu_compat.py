"""The reference's generated-library ABI (initializeArrays / computeMonodomain) exported by the library,
driven the way FastMonodomainSolverBase::computeMonodomainGpu drives it (fast_monodomain_solver_gpu.tpp:1010-1118),
against the oracle with the centre clamp rule of the reference's GPU code."""
import ctypes as C
import math

import numpy as np
import pytest

import helpers as H
from opendihu_b200 import _native as N

pytestmark = pytest.mark.gpu


def _tss_n(span, dt):
    return max(1, int(math.ceil(span / dt - 0.1)))


def test_compat_abi_matches_oracle():
    L = N.lib()
    n_fibers, n_per = 3, 301
    sysm = H.c1_system(n_fibers=n_fibers, n_nodes=n_per, end_time=1.0, clamp_rule="center")
    sysm.element_lengths = np.full_like(sysm.element_lengths, float(np.float32(0.01)))
    H.complete(sysm)
    ref, _, _, n_ref = H.run_oracle(sysm.copy())
    assert L.fdm_compat_configure(0, n_fibers, n_per, 1, 1, 1, 0, 0, 2, 0, 0, 0, 1) == 0, L.fdm_last_error(None)
    states_one = np.ascontiguousarray(H.initial_states(H.HH, 1)[:, 0])
    alg_idx = np.zeros(1, np.int32)
    st_idx = np.array([0, 1], np.int32)
    firing = C.create_string_buffer(b"\x01", 1)
    jitter = np.zeros(1)
    mu = np.zeros(n_fibers, np.int32)
    center = np.full(n_fibers, n_per // 2, np.int32)
    freq = np.full(n_fibers, 0.1)
    rep = np.full(n_fibers, 0.1)
    beg = np.zeros(n_fibers)
    last = beg - 1e-13 - 1.0 / freq
    p = N.ptr
    L.initializeArrays(p(states_one, C.c_double), p(alg_idx, C.c_int), p(st_idx, C.c_int), firing,
                       p(jitter, C.c_double), p(mu, C.c_int), p(center, C.c_int), p(last, C.c_double),
                       p(freq, C.c_double), p(rep, C.c_double), p(beg, C.c_double))
    n = n_fibers * n_per
    params = np.zeros(n, np.float32)
    lengths = np.full(n_fibers * (n_per - 1), 0.01, np.float32)
    out_states = np.zeros((2, n))
    out_alg = np.zeros(1)
    # RepeatedCall over [0, 1] with dt 1e-3, one Strang step per call (repeated_call.tpp:59-75)
    t0, t1, dtr = 0.0, 1.0, 1e-3
    nrc = _tss_n(t1 - t0, dtr)
    dtr = (t1 - t0) / nrc
    t = t0
    for k in range(nrc):
        dts = (t + dtr) - t
        n0 = _tss_n((t + 0.5 * dts) - t, 1e-4)
        dt0 = ((t + 0.5 * dts) - t) / n0
        dt1 = ((t + dts) - t) / _tss_n(dts, 1e-3)
        L.computeMonodomain(p(params, C.c_float), p(out_alg, C.c_double), p(out_states, C.c_double),
                            p(lengths, C.c_float), t, dts, 1, dt0, n0, dt1, 1, 3.828 / 500, 20.0)
        t = t0 + (k + 1) / nrc * (t1 - t0)
    assert nrc == n_ref
    assert np.max(np.abs(out_states[0] - ref[0])) <= 1e-6
    assert np.max(np.abs(out_states[1] - ref[1])) <= 1e-8
    assert L.fdm_compat_release() == 0
