"""Shared test helpers: build problems, convert them to oracle runs, compare results."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from opendihu_b200 import solver as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

HH = "hodgkin_huxley_1952"
SHORTEN = "shorten_ocallaghan_davidson_soboleva_2007"

#: raw CONSTANTS of the parameter slots of the built variants (I_Stim, g_Na, g_K for HH; ALGEBRAIC[32], l_hs)
HH_DEFAULT_PARAMS = np.array([0.0, 120.0, 36.0])


def default_parameters(model, n_nodes):
    ns, na, npar, init = O.model_info(model)
    if model == HH:
        d = HH_DEFAULT_PARAMS
    else:
        d = np.array([0.0, 1.0])
    return np.repeat(d[:, None], n_nodes, axis=1)


def initial_states(model, n_nodes):
    ns, na, npar, init = O.model_info(model)
    return np.repeat(init[:, None], n_nodes, axis=1)


def complete(system: S.FiberSystem) -> S.FiberSystem:
    """Fill parameters/states with the model defaults if missing."""
    if system.parameters is None:
        system.parameters = default_parameters(system.model, system.n_nodes)
    if system.states is None:
        system.states = initial_states(system.model, system.n_nodes)
    return system


def oracle_spec(system: S.FiberSystem, n_threads: int = 0, trace_nodes=(), trace_capacity: int = 0):
    complete(system)
    return {
        "model": system.model, "fiber_offsets": system.fiber_offsets, "element_lengths": system.element_lengths,
        "prefactor": system.prefactor, "parameters": system.parameters,
        "diffusion_scheme": S.SCHEMES[system.diffusion_scheme],
        "approx_exp": int(system.approximate_exponential_function), "clamp_rule": S.CLAMP_RULES[system.clamp_rule],
        "vc_width": system.vc_width, "n_ranks": system.n_ranks,
        "stimulus_mode": S.STIMULUS_MODES[system.stimulus_mode], "stimulus_parameter": system.stimulus_parameter,
        "stimulus_value": system.stimulus_value, "value_for_stimulated_point": system.value_for_stimulated_point,
        "firing_events": system.firing_events, "motor_unit_no": system.motor_unit_no,
        "stimulation_point_index": system.stimulation_point_index, "call_frequency": system.call_frequency,
        "repeat_after_first_call": system.repeat_after_first_call, "call_enable_begin": system.call_enable_begin,
        "jitter": system.jitter if system.jitter is not None else np.zeros((system.n_fibers, 0)),
        "t_start": system.start_time, "t_end": system.end_time, "dt_repeated_call": system.dt_repeated_call,
        "dt_splitting": system.dt_splitting, "dt_0d": system.dt_0d, "dt_1d": system.dt_1d,
        "n_threads": n_threads or (os.cpu_count() or 1),
        "algebraic_indices": list(system.algebraics_for_transfer),
        "trace_nodes": list(trace_nodes), "trace_capacity": trace_capacity,
        "only_if_stimulated": bool(getattr(system, "only_compute_if_has_been_stimulated", False)),
        "equilibrium": bool(getattr(system, "skip_close_to_equilibrium", False)),
    }


def run_oracle(system: S.FiberSystem, n_threads: int = 0, trace_nodes=(), trace_capacity: int = 0):
    """Returns (states [s][node], algebraics [k][node], trace [step][k], n_split_steps)."""
    spec = oracle_spec(system, n_threads, trace_nodes, trace_capacity)
    run = O.OracleRun(spec)
    st = np.ascontiguousarray(system.states, np.float64).copy()
    n = run.run(st)
    return st, run.algebraics[:len(system.algebraics_for_transfer)].copy(), run.trace[:min(n, trace_capacity)].copy(), n


def activation_times(trace: np.ndarray, dt: float, threshold: float = 0.0):
    """First split step index (times dt) at which each traced node crosses `threshold` upwards; nan if never."""
    out = np.full(trace.shape[1], np.nan)
    for k in range(trace.shape[1]):
        above = np.nonzero(trace[:, k] > threshold)[0]
        if len(above):
            out[k] = (above[0] + 1) * dt
    return out


def c1_system(n_fibers=16, n_nodes=1481, end_time=10.0, **kw) -> S.FiberSystem:
    """Hodgkin-Huxley fibers of the plain-method benchmark configuration: dx 0.01 cm,
    prefactor sigma/(Am*Cm) = 3.828/(500*1), Heun dt 1e-4, Strang/IE dt 1e-3, clamp stimulus every 10 ms."""
    return S.uniform_fibers(HH, [n_nodes] * n_fibers, 0.01, 3.828 / (500 * 1.0), call_frequency=0.1,
                            repeat_after_first_call=0.1, call_enable_begin=0.0, end_time=end_time,
                            dt_0d=1e-4, dt_1d=1e-3, dt_splitting=1e-3, dt_repeated_call=1e-3, **kw)
