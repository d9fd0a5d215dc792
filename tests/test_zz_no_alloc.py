"""The allocation-free diffusion solve against the allocating one.

fdm_diffusion_solve_noalloc is for callers that cannot allocate device memory while they run (their own
memory pool owns the GPU, or a stepping loop must not synchronize on cudaMalloc/cudaFree); it takes its
scratch from an array compiled into the library.  It runs the same kernels as fdm_diffusion_solve on the
same inputs, so the results must be identical bit for bit, call after call, although the array keeps the
previous call's contents.  Both diffusion kernels are covered: a CTA per fiber below 592 fibers and a warp
per fiber from 592 fibers on.  This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from opendihu_b200 import _native as N

pytestmark = pytest.mark.gpu

#: fibers from which launch_diffusion switches from a CTA per fiber to a warp per fiber
WARP_KERNEL_MIN_FIBERS = 4 * 148


def _device_problem(torch, n_fibers=40, lengths=(300, 3000), seed=11):
    rng = np.random.default_rng(seed)
    lengths = rng.integers(lengths[0], lengths[1], size=n_fibers)
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
    return fn(n_fibers, n, C.c_void_p(off.data_ptr()), C.c_void_p(h.data_ptr()), C.c_void_p(pf.data_ptr()), dt,
              scheme, C.c_void_p(vm.data_ptr()), None)


@pytest.mark.parametrize("fibers,lengths", [(40, (300, 3000)), (WARP_KERNEL_MIN_FIBERS + 8, (300, 400))],
                         ids=["cta_per_fiber", "warp_per_fiber"])
@pytest.mark.parametrize("scheme", [0, 1], ids=["IE", "CN"])
def test_noalloc_diffusion_matches_allocating_solve_twice(scheme, fibers, lengths):
    import torch
    L = N.lib()
    n_fibers, n, off, h, pf, vm0, dev = _device_problem(torch, n_fibers=fibers, lengths=lengths)
    a = torch.from_numpy(vm0.copy()).to(dev)
    b = torch.from_numpy(vm0.copy()).to(dev)
    for call in range(2):
        N.check(_call(L.fdm_diffusion_solve, n_fibers, n, off, h, pf, 1e-3, scheme, a))
        N.check(_call(L.fdm_diffusion_solve_noalloc, n_fibers, n, off, h, pf, 1e-3, scheme, b))
        torch.cuda.synchronize()
        va, vb = a.cpu().numpy(), b.cpu().numpy()
        assert np.all(np.isfinite(vb))
        # same kernels, same inputs: identical bits
        assert np.array_equal(va.view(np.int64), vb.view(np.int64)), f"call {call}: {np.max(np.abs(va - vb))}"
        assert np.max(np.abs(va - vm0)) > 0  # the solve did something


def test_noalloc_rejects_sizes_beyond_maximum():
    import torch
    L = N.lib()
    n_fibers, n, off, h, pf, vm0, dev = _device_problem(torch, n_fibers=3)
    vm = torch.from_numpy(vm0).to(dev)
    rc = _call(L.fdm_diffusion_solve_noalloc, n_fibers, N.NOALLOC_MAX_NODES + 1, off, h, pf, 1e-3, 0, vm)
    assert rc == N.FDM_ERR_ARG
    assert b"FDM_NOALLOC_MAX_NODES" in L.fdm_last_error(None)


def test_noalloc_rejects_offsets_beyond_n_nodes():
    """Offsets whose last entry passes n_nodes would index past the library's array: refused, nothing runs."""
    import torch
    L = N.lib()
    n_fibers, n, off, h, pf, vm0, dev = _device_problem(torch, n_fibers=3)
    vm = torch.from_numpy(vm0.copy()).to(dev)
    rc = _call(L.fdm_diffusion_solve_noalloc, n_fibers, n - 1, off, h, pf, 1e-3, 0, vm)
    assert rc == N.FDM_ERR_ARG
    assert b"fiber offsets" in L.fdm_last_error(None)
    assert np.array_equal(vm.cpu().numpy(), vm0)
