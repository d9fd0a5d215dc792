"""Differentiation extension: gradients of a Vm-trace loss with respect to per-fiber conductivity and
per-node parameters (e.g. channel conductances), through the hand-written discrete adjoint of the FP64
Strang step (libfdm_b200: fdm_adjoint_forward / fdm_adjoint_backward), exposed to PyTorch as a
``torch.autograd.Function``.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from .solver import FastMonodomainSolver, FiberSystem, model_sizes


class AdjointEngine:
    """Holds one FP64 split solver; ``forward(prefactor, parameters)`` runs the checkpointed forward and
    returns the sensor trace, ``backward(dL/dtrace)`` the gradients."""

    def __init__(self, system: FiberSystem, sensor_nodes: Sequence[int], checkpoint_every: int = 100,
                 device: int = 0):
        self.system = system.copy()
        ns, na, npar, init, defaults = model_sizes(self.system.model)
        if self.system.states is None:
            self.system.states = np.repeat(init[:, None], self.system.n_nodes, axis=1)
        if self.system.parameters is None:
            self.system.parameters = np.repeat(defaults[:, None], self.system.n_nodes, axis=1)
        self.initial_states = np.array(self.system.states, np.float64)
        self.sensor_nodes = np.asarray(sensor_nodes, np.int64)
        self.checkpoint_every = int(checkpoint_every)
        self.solver = FastMonodomainSolver(self.system, method="split", precision="fp64", device=device)
        self.solver.initialize()

    def forward(self, prefactor: np.ndarray, parameters: np.ndarray) -> np.ndarray:
        s = self.solver
        s.set_prefactor(np.asarray(prefactor, np.float64))
        s.set_parameters(np.asarray(parameters, np.float64))
        s.set_states(self.initial_states)
        s.rewind()
        sysm = self.system
        return s.adjoint_forward(sysm.start_time, sysm.end_time, self.checkpoint_every, self.sensor_nodes)

    def backward(self, trace_grad: np.ndarray):
        return self.solver.adjoint_backward(trace_grad)

    def close(self):
        self.solver.close()


def _torch_function():
    import torch

    class StrangTrace(torch.autograd.Function):
        """trace = StrangTrace.apply(prefactor[n_fibers], parameters[n_params, n_nodes], engine)

        The trace is Vm at the engine's sensor nodes after every Strang step of [start_time, end_time];
        backward returns dL/dprefactor and dL/dparameters from the discrete adjoint (FP64)."""

        @staticmethod
        def forward(ctx, prefactor, parameters, engine):
            trace = engine.forward(prefactor.detach().cpu().double().numpy(),
                                   parameters.detach().cpu().double().numpy())
            ctx.engine = engine
            ctx.device = prefactor.device
            return torch.from_numpy(trace).to(prefactor.device)

        @staticmethod
        def backward(ctx, grad_trace):
            g = ctx.engine.backward(grad_trace.detach().cpu().double().numpy())
            return (torch.from_numpy(g["prefactor"]).to(ctx.device),
                    torch.from_numpy(g["parameters"]).to(ctx.device), None)

    return StrangTrace


_FN = None


def strang_trace(prefactor, parameters, engine: AdjointEngine):
    """Differentiable sensor trace (torch tensors in, torch tensor out)."""
    global _FN
    if _FN is None:
        _FN = _torch_function()
    return _FN.apply(prefactor, parameters, engine)
