"""The allocation-free diffusion solve against the allocating one.

fdm_diffusion_solve_noalloc is for callers that cannot allocate device memory while they run (their own
memory pool owns the GPU, or a stepping loop must not synchronize on cudaMalloc/cudaFree); it takes its
scratch from an array compiled into the library.  It must give the same result as fdm_diffusion_solve on
the same inputs, call after call, although the array keeps the previous call's contents.  This file is
collected last so that a run stopping at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from opendihu_b200 import _native as N

pytestmark = pytest.mark.gpu

#: the FP64 tolerance the parity tests use for Vm (mV); the two entry points run the same kernels
VM_TOL_FP64 = 1e-6


def _device_problem(torch, n_fibers=40, seed=11):
    rng = np.random.default_rng(seed)
    lengths = rng.integers(300, 3000, size=n_fibers)
    off = np.zeros(n_fibers + 1, np.int64)
    off[1:] = np.cumsum(lengths)
    n = int(off[-1])
    assert n <= N.NOALLOC_MAX_NODES
    h = rng.uniform(0.008, 0.012, size=n - n_fibers)
    pf = rng.uniform(2.5, 5.0, size=n_fibers) / 500.0
    vm = rng.uniform(-80.0, 30.0, size=n)
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(a).to(dev)
    return n_fibers, n, t(off), t(h), t(pf), vm, dev


def _call(fn, n_fibers, n, off, h, pf, dt, scheme, vm):
    rc = fn(n_fibers, n, C.c_void_p(off.data_ptr()), C.c_void_p(h.data_ptr()), C.c_void_p(pf.data_ptr()), dt,
            scheme, C.c_void_p(vm.data_ptr()), None)
    N.check(rc)


@pytest.mark.parametrize("scheme", [0, 1])
def test_noalloc_diffusion_matches_allocating_solve_twice(scheme):
    import torch
    L = N.lib()
    n_fibers, n, off, h, pf, vm0, dev = _device_problem(torch)
    a = torch.from_numpy(vm0.copy()).to(dev)
    b = torch.from_numpy(vm0.copy()).to(dev)
    for call in range(2):
        _call(L.fdm_diffusion_solve, n_fibers, n, off, h, pf, 1e-3, scheme, a)
        _call(L.fdm_diffusion_solve_noalloc, n_fibers, n, off, h, pf, 1e-3, scheme, b)
        torch.cuda.synchronize()
        va, vb = a.cpu().numpy(), b.cpu().numpy()
        assert np.all(np.isfinite(vb))
        assert np.max(np.abs(va - vb)) <= VM_TOL_FP64, f"call {call}: {np.max(np.abs(va - vb))}"
        assert np.max(np.abs(va - vm0)) > 0  # the solve did something


def test_noalloc_rejects_sizes_beyond_maximum():
    import torch
    L = N.lib()
    n_fibers, n, off, h, pf, vm0, dev = _device_problem(torch, n_fibers=3)
    vm = torch.from_numpy(vm0).to(dev)
    rc = L.fdm_diffusion_solve_noalloc(n_fibers, N.NOALLOC_MAX_NODES + 1, C.c_void_p(off.data_ptr()),
                                       C.c_void_p(h.data_ptr()), C.c_void_p(pf.data_ptr()), 1e-3, 0,
                                       C.c_void_p(vm.data_ptr()), None)
    assert rc == N.FDM_ERR_ARG
    assert b"FDM_NOALLOC_MAX_NODES" in L.fdm_last_error(None)
