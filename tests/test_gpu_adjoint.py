"""The hand-written adjoint (CUDA, FP64) against an FP64 reference gradient (torch autograd through an
independent implementation of the same discrete Strang map, itself checked against the oracle) and against
central finite differences of the CUDA forward."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import helpers as H
import torch_reference as TR
from opendihu_b200 import adjoint as ADJ
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def _problem(scheme="ImplicitEuler", rule="vc", end_time=0.15, seed=3, nodes=21):
    sysm = H.c1_system(n_fibers=2, n_nodes=nodes, end_time=end_time, diffusion_scheme=scheme, clamp_rule=rule)
    H.complete(sysm)
    rng = np.random.default_rng(seed)
    sysm.prefactor = rng.uniform(2.5, 5.0, size=2) / 500
    sysm.parameters = WL.hh_parameters(sysm, rng.uniform(0.8, 1.2, 2), rng.uniform(0.8, 1.2, 2))
    sensors = np.array([0, 5, 10, nodes + 3, 2 * nodes - 1])
    return sysm, sensors, rng


@pytest.mark.parametrize("scheme,rule,ck", [("ImplicitEuler", "vc", 7), ("CrankNicolson", "center", 1),
                                            ("CrankNicolson", "vc", 1000)])
def test_adjoint_matches_autograd_reference(scheme, rule, ck):
    sysm, sensors, rng = _problem(scheme, rule)
    eng = ADJ.AdjointEngine(sysm, sensors, checkpoint_every=ck)
    try:
        trace = eng.forward(sysm.prefactor, sysm.parameters)
        w = rng.standard_normal(trace.shape)
        g = eng.backward(w)
        first, cnt, _ = eng.solver.clamp_nodes()
    finally:
        eng.close()
    pf = torch.tensor(sysm.prefactor, requires_grad=True)
    P = torch.tensor(sysm.parameters, requires_grad=True)
    tr, _ = TR.forward(sysm, pf, P, sensors, first, cnt)
    (torch.tensor(w) * tr).sum().backward()
    np.testing.assert_allclose(trace, tr.detach().numpy(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(g["prefactor"], pf.grad.numpy(), rtol=1e-7, atol=1e-9 * np.abs(pf.grad.numpy()).max())
    gp = P.grad.numpy()
    np.testing.assert_allclose(g["parameters"], gp, rtol=1e-7, atol=1e-9 * np.abs(gp).max())


def test_adjoint_central_differences_and_autograd_function():
    sysm, sensors, rng = _problem(end_time=0.3)
    eng = ADJ.AdjointEngine(sysm, sensors, checkpoint_every=50)
    target = None
    try:
        base = eng.forward(sysm.prefactor, sysm.parameters)
        target = base + rng.standard_normal(base.shape) * 0.5
        pf = torch.tensor(sysm.prefactor, requires_grad=True)
        P = torch.tensor(sysm.parameters, requires_grad=True)
        tr = ADJ.strang_trace(pf, P, eng)
        loss = ((tr - torch.tensor(target)) ** 2).sum()
        loss.backward()

        def L(pfv, Pv):
            t = eng.forward(pfv, Pv)
            return float(((t - target) ** 2).sum())
        h = 1e-6
        for f in range(2):
            d = np.zeros(2)
            d[f] = h * sysm.prefactor[f]
            fd = (L(sysm.prefactor + d, sysm.parameters) - L(sysm.prefactor - d, sysm.parameters)) / (2 * d[f])
            assert abs(fd - pf.grad[f].item()) <= 1e-4 * abs(fd) + 1e-6, (f, fd, pf.grad[f].item())
        # g_Na scale of fiber 1: all nodes of the fiber move together
        lengths = np.diff(sysm.fiber_offsets)
        mask = np.repeat(np.arange(2) == 1, lengths)
        dP = np.zeros_like(sysm.parameters)
        dP[1, mask] = h * 120.0
        fd = (L(sysm.prefactor, sysm.parameters + dP) - L(sysm.prefactor, sysm.parameters - dP)) / (2 * h)
        ad = float((P.grad.numpy()[1, mask] * 120.0).sum())
        assert abs(fd - ad) <= 1e-4 * abs(fd) + 1e-6, (fd, ad)
    finally:
        eng.close()


def test_solver_continues_after_adjoint():
    sysm, sensors, rng = _problem(end_time=0.2)
    with S.FastMonodomainSolver(sysm.copy(), method="split", precision="fp64") as slv:
        slv.adjoint_forward(0.0, 0.2, 30, sensors)
        a = slv.states()
        slv.adjoint_backward(np.ones((200, len(sensors))))
        b = slv.states()
    np.testing.assert_array_equal(a, b)
    ref, _, _, _ = H.run_oracle(sysm.copy())
    assert np.max(np.abs(a[0] - ref[0])) <= 1e-6


def test_shorten_adjoint_central_differences():
    """The 56-state Shorten model through the same adjoint (generated vector-Jacobian product of its
    right-hand side): prefactor and parameter gradients against central differences of the forward run."""
    sysm = S.uniform_fibers(H.SHORTEN, [31, 25], 0.01, 3.828 / (500 * 0.58), call_frequency=0.1,
                            repeat_after_first_call=0.1, end_time=0.02, dt_0d=1e-5, dt_1d=5e-4, dt_splitting=5e-4,
                            dt_repeated_call=5e-4)
    H.complete(sysm)
    sensors = np.array([0, 7, 15, 31 + 4, 55])
    rng = np.random.default_rng(8)
    eng = ADJ.AdjointEngine(sysm, sensors, checkpoint_every=7)
    try:
        base = eng.forward(sysm.prefactor, sysm.parameters)
        w = rng.standard_normal(base.shape)
        g = eng.backward(w)

        def L(pfv, Pv):
            return float((w * eng.forward(pfv, Pv)).sum())
        h = 1e-6
        for f in range(2):
            d = np.zeros(2)
            d[f] = h * sysm.prefactor[f]
            fd = (L(sysm.prefactor + d, sysm.parameters) - L(sysm.prefactor - d, sysm.parameters)) / (2 * d[f])
            assert abs(fd - g["prefactor"][f]) <= 1e-4 * abs(fd) + 1e-8, (f, fd, g["prefactor"][f])
        lengths = np.diff(sysm.fiber_offsets)
        mask = np.repeat(np.arange(2) == 1, lengths)
        p = sysm.parameters.shape[0] - 1
        scale = max(abs(float(sysm.parameters[p, mask][0])), 1.0)
        dP = np.zeros_like(sysm.parameters)
        dP[p, mask] = h * scale
        fd = (L(sysm.prefactor, sysm.parameters + dP) - L(sysm.prefactor, sysm.parameters - dP)) / (2 * h * scale)
        ad = float(g["parameters"][p, mask].sum())
        assert abs(fd - ad) <= 1e-4 * abs(fd) + 1e-8, (fd, ad)
    finally:
        eng.close()


@pytest.mark.slow
def test_adjoint_at_configuration_size_against_central_differences():
    """The differentiation configuration as specified: 256 HH fibers x 1481 nodes, per-fiber sigma ~ U[2.5, 5]
    and g_Na, g_K scales ~ U[0.8, 1.2] (seed 1), loss = sum of squared Vm differences at 32 sensors per fiber over
    20 ms against the trace of a second parameter set (seed 2), checkpoint every 100 Strang steps.  The adjoint
    gradient of sigma, g_Na scale and g_K scale of two fibers against central differences with relative step
    h = 1e-6 of the CUDA FP64 forward."""
    dsys, sigma, s_na, s_k, sensors = WL.differentiation_hh(end_time=20.0, seed=1)
    _, sigma2, s_na2, s_k2, _ = WL.differentiation_hh(end_time=20.0, seed=2)
    eng = ADJ.AdjointEngine(dsys, sensors, checkpoint_every=100)
    lengths = np.diff(dsys.fiber_offsets)
    fiber_of = np.repeat(np.arange(dsys.n_fibers), lengths)
    try:
        target = eng.forward(sigma2 / (WL.AM * WL.CM), WL.hh_parameters(dsys, s_na2, s_k2))

        def loss(sig, sna, sk):
            tr = eng.forward(sig / (WL.AM * WL.CM), WL.hh_parameters(dsys, sna, sk))
            return float(((tr - target) ** 2).sum()), tr

        L0, tr = loss(sigma, s_na, s_k)
        assert tr.shape == (20000, 256 * 32)
        g = eng.backward(2.0 * (tr - target))
        g_sigma = g["prefactor"] / (WL.AM * WL.CM)
        g_na = np.bincount(fiber_of, g["parameters"][1] * 120.0, minlength=dsys.n_fibers)
        g_k = np.bincount(fiber_of, g["parameters"][2] * 36.0, minlength=dsys.n_fibers)
        for f in (0, 255):
            for name, vec, grad in (("sigma", sigma, g_sigma), ("g_Na", s_na, g_na), ("g_K", s_k, g_k)):
                h = 1e-6 * vec[f]
                plus, minus = vec.copy(), vec.copy()
                plus[f] += h
                minus[f] -= h
                args_p = {"sigma": (plus, s_na, s_k), "g_Na": (sigma, plus, s_k), "g_K": (sigma, s_na, plus)}[name]
                args_m = {"sigma": (minus, s_na, s_k), "g_Na": (sigma, minus, s_k), "g_K": (sigma, s_na, minus)}[name]
                fd = (loss(*args_p)[0] - loss(*args_m)[0]) / (2 * h)
                print(name, f, grad[f], fd)
                assert abs(grad[f] - fd) <= 1e-4 * max(abs(fd), 1e-6 * abs(L0)), (name, f, grad[f], fd)
    finally:
        eng.close()
