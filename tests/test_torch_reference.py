"""The torch FP64 reference of the discrete forward agrees with the oracle (so that its autograd gradient can
serve as the reference gradient of the CUDA adjoint)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import helpers as H
import torch_reference as TR


@pytest.mark.parametrize("scheme,rule", [("ImplicitEuler", "vc"), ("CrankNicolson", "center")])
def test_torch_forward_matches_oracle(scheme, rule):
    sysm = H.c1_system(n_fibers=2, n_nodes=21, end_time=0.15, diffusion_scheme=scheme, clamp_rule=rule)
    H.complete(sysm)
    rng = np.random.default_rng(0)
    sysm.prefactor = rng.uniform(2.5, 5.0, size=2) / 500
    sensors = [0, 5, 10, 21 + 7, 41]
    ref, _, tr_ref, n = H.run_oracle(sysm.copy(), trace_nodes=sensors, trace_capacity=1000)
    first, cnt = H.O.OracleRun(H.oracle_spec(sysm.copy())).vc_clamp_nodes()
    if rule == "center":
        c = sysm.stimulation_point_index
        first = np.asarray(sysm.fiber_offsets[:-1]) + c - 1
        cnt = np.full(2, 3)
    pf = torch.tensor(sysm.prefactor)
    P = torch.tensor(sysm.parameters)
    tr, y = TR.forward(sysm, pf, P, sensors, first, cnt)
    assert tr.shape[0] == n
    np.testing.assert_allclose(tr.detach().numpy(), tr_ref[:n], rtol=0, atol=1e-9)
    np.testing.assert_allclose(y[0].detach().numpy(), ref[0], rtol=0, atol=1e-9)
