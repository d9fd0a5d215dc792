"""onlyComputeIfHasBeenStimulated on the GPU: split and fused paths against the oracle's buffer-order
restatement (vc and centre rules, FP64 and FP32 reaction, window sizes), and the adjoint of the gated
forward against the torch autograd reference."""
import numpy as np
import pytest

import helpers as H
import test_gpu_parity as GP
from opendihu_b200 import _native as N
from opendihu_b200 import adjoint as ADJ
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def _system(rule="vc", end_time=1.2):
    # four fibers of uneven length; motor unit 1 never fires; fibers 2 and 3 start firing later
    s = WL.batched_hh(n_fibers=4, min_nodes=40, max_nodes=90, seed=7, end_time=end_time, clamp_rule=rule)
    s.firing_events = np.array([[1, 0, 1, 1]], np.uint8)
    s.motor_unit_no = np.array([0, 1, 2, 3], np.int32)
    s.call_enable_begin = np.array([0.0, 0.0, 0.35, 0.8123])
    s.only_compute_if_has_been_stimulated = True
    return H.complete(s)


@pytest.mark.parametrize("method,rule", [("split", "vc"), ("fused", "vc"), ("split", "center"), ("fused", "center")])
def test_fp64_matches_oracle(method, rule):
    GP.compare(_system(rule), method, "fp64", GP.VM_TOL_FP64, 1e-8)


def test_fp32_fused_within_01mV():
    GP.compare(_system(), "fused", "fp32", GP.VM_TOL_FP32, 1e-3)


@pytest.mark.parametrize("method", ["split", "fused"])
def test_window_sizes_do_not_change_results(method):
    s = _system(end_time=0.9)
    outs = [GP.run_gpu(s.copy(), method, steps_per_launch=k)[0] for k in (1, 7, 100)]
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])


def test_adjoint_of_the_gated_forward():
    torch = pytest.importorskip("torch")
    import torch_reference as TR
    sysm = H.c1_system(n_fibers=2, n_nodes=21, end_time=0.12)
    H.complete(sysm)
    sysm.firing_events = np.array([[1, 0]], np.uint8)
    sysm.motor_unit_no = np.array([0, 1], np.int32)
    sysm.only_compute_if_has_been_stimulated = True
    rng = np.random.default_rng(4)
    sysm.prefactor = rng.uniform(2.5, 5.0, size=2) / 500
    sysm.parameters = WL.hh_parameters(sysm, rng.uniform(0.8, 1.2, 2), rng.uniform(0.8, 1.2, 2))
    sensors = np.array([0, 5, 10, 24, 41])
    eng = ADJ.AdjointEngine(sysm, sensors, checkpoint_every=7)
    try:
        trace = eng.forward(sysm.prefactor, sysm.parameters)
        w = rng.standard_normal(trace.shape)
        g = eng.backward(w)
        first, cnt, _ = eng.solver.clamp_nodes()
    finally:
        eng.close()
    codes = N.select_gate_codes(S.CLAMP_RULES[sysm.clamp_rule], sysm.vc_width, sysm.n_ranks, sysm.fiber_offsets,
                                sysm.stimulation_point_index)
    pf = torch.tensor(sysm.prefactor, requires_grad=True)
    P = torch.tensor(sysm.parameters, requires_grad=True)
    tr, _ = TR.forward(sysm, pf, P, sensors, first, cnt, gate_codes=codes)
    (torch.tensor(w) * tr).sum().backward()
    np.testing.assert_allclose(trace, tr.detach().numpy(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(g["prefactor"], pf.grad.numpy(), rtol=1e-7, atol=1e-9 * np.abs(pf.grad.numpy()).max())
    gp = P.grad.numpy()
    np.testing.assert_allclose(g["parameters"], gp, rtol=1e-7, atol=1e-9 * np.abs(gp).max())
    # fiber 1 is never stimulated: its nodes attributed to it carry no parameter gradient
    att = codes >> 2
    assert np.all(g["parameters"][:, att == 1] == 0.0)
