"""ctypes wrapper of the CPU oracle (liboracle.so, built from fdm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, never by the product package.  The oracle restates the reference's "vc"
FastMonodomainSolver in plain FP64 C; see fdm_oracle.c for the reference lines it follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

MODELS = {"hodgkin_huxley_1952": 0, "shorten_ocallaghan_davidson_soboleva_2007": 1}


def build(force: bool = False) -> str:
    """Compile liboracle.so (gcc, no FMA contraction, OpenMP for the threaded baseline)."""
    src = os.path.join(HERE, "fdm_oracle.c")
    deps = [src, os.path.join(HERE, "oracle_math.h")] + [
        os.path.join(HERE, "generated", f) for f in os.listdir(os.path.join(HERE, "generated"))]
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(d) for d in deps):
        return LIB_PATH
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           "-o", LIB_PATH, src, "-lm"]
    subprocess.check_call(cmd, cwd=HERE)
    return LIB_PATH


class Problem(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("n_fibers", C.c_int),
        ("fiber_offsets", C.POINTER(C.c_int64)), ("element_lengths", C.POINTER(C.c_double)),
        ("prefactor", C.POINTER(C.c_double)), ("parameters", C.POINTER(C.c_double)),
        ("diffusion_scheme", C.c_int), ("approx_exp", C.c_int), ("clamp_rule", C.c_int),
        ("vc_width", C.c_int), ("n_ranks", C.c_int), ("stimulus_mode", C.c_int),
        ("stimulus_parameter", C.c_int), ("stimulus_value", C.c_double),
        ("value_for_stimulated_point", C.c_double),
        ("firing_events", C.POINTER(C.c_uint8)), ("firing_rows", C.c_int), ("firing_cols", C.c_int),
        ("motor_unit_no", C.POINTER(C.c_int)), ("stimulation_point_index", C.POINTER(C.c_int)),
        ("call_frequency", C.POINTER(C.c_double)), ("repeat_after_first_call", C.POINTER(C.c_double)),
        ("call_enable_begin", C.POINTER(C.c_double)), ("jitter", C.POINTER(C.c_double)),
        ("n_jitter", C.c_int),
        ("t_start", C.c_double), ("t_end", C.c_double),
        ("dt_repeated_call", C.c_double), ("dt_splitting", C.c_double), ("dt_0d", C.c_double),
        ("dt_1d", C.c_double), ("n_threads", C.c_int),
        ("n_algebraics_out", C.c_int), ("algebraic_indices", C.POINTER(C.c_int)),
        ("algebraics_out", C.POINTER(C.c_double)),
        ("n_trace_nodes", C.c_int), ("trace_nodes", C.POINTER(C.c_int64)), ("trace", C.POINTER(C.c_double)),
        ("trace_capacity", C.c_int64),
        ("only_if_stimulated", C.c_int), ("has_been_stimulated", C.POINTER(C.c_int)),
        ("equilibrium", C.c_int), ("eq_status", C.POINTER(C.c_uint8)), ("eq_counter", C.POINTER(C.c_int)),
        ("pad_states", C.POINTER(C.c_double)),
        ("currently_stimulating", C.POINTER(C.c_int)), ("log_times", C.POINTER(C.c_double)),
        ("log_fibers", C.POINTER(C.c_int)), ("log_capacity", C.c_int64), ("log_count", C.POINTER(C.c_int64)),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.oracle_run.restype = C.c_int64
        _lib.oracle_run.argtypes = [C.POINTER(Problem), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_int)]
        _lib.oracle_model_info.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                           C.POINTER(C.c_double)]
        _lib.oracle_rates.argtypes = [C.c_int, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
        _lib.oracle_explicit_euler_cell.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                    C.c_double, C.c_double, C.c_int, C.c_int]
        _lib.oracle_vc_clamp_nodes.argtypes = [C.POINTER(Problem), C.POINTER(C.c_int64), C.POINTER(C.c_int)]
        _lib.oracle_stimulation_init.argtypes = [C.POINTER(Problem), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                 C.POINTER(C.c_int)]
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def model_info(model: str):
    ns, na, npar = C.c_int(), C.c_int(), C.c_int()
    init = np.zeros(64)
    lib().oracle_model_info(MODELS[model], C.byref(ns), C.byref(na), C.byref(npar), _p(init, C.c_double))
    return ns.value, na.value, npar.value, init[:ns.value].copy()


def rates(model: str, states, params, t: float = 0.0, approx: bool = False):
    ns, na, npar, _ = model_info(model)
    s = np.ascontiguousarray(states, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64)
    r = np.zeros(ns)
    a = np.zeros(na)
    lib().oracle_rates(MODELS[model], t, _p(s, C.c_double), _p(p, C.c_double), _p(r, C.c_double),
                       _p(a, C.c_double), int(approx))
    return r, a


def explicit_euler_cell(model: str, states, params, dt: float, n_steps: int, t0: float = 0.0,
                        approx: bool = False) -> np.ndarray:
    s = np.array(states, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64)
    lib().oracle_explicit_euler_cell(MODELS[model], _p(s, C.c_double), _p(p, C.c_double), t0, dt, n_steps,
                                     int(approx))
    return s


class OracleRun:
    """Holds the arrays of one oracle problem (keeps them alive while the C side uses them)."""

    def __init__(self, spec: Dict):
        self.spec = spec
        self.keep = []
        p = Problem()
        a = self._arr
        p.model = MODELS[spec["model"]]
        offsets = a(spec["fiber_offsets"], np.int64)
        p.n_fibers = len(offsets) - 1
        p.fiber_offsets = _p(offsets, C.c_int64)
        p.element_lengths = _p(a(spec["element_lengths"], np.float64), C.c_double)
        p.prefactor = _p(a(spec["prefactor"], np.float64), C.c_double)
        p.parameters = _p(a(spec["parameters"], np.float64), C.c_double)
        p.diffusion_scheme = int(spec.get("diffusion_scheme", 0))
        p.approx_exp = int(spec.get("approx_exp", 0))
        p.clamp_rule = int(spec.get("clamp_rule", 0))
        p.vc_width = int(spec.get("vc_width", 4))
        p.n_ranks = int(spec.get("n_ranks", 1))
        p.stimulus_mode = int(spec.get("stimulus_mode", 0))
        p.stimulus_parameter = int(spec.get("stimulus_parameter", 0))
        p.stimulus_value = float(spec.get("stimulus_value", 0.0))
        p.value_for_stimulated_point = float(spec.get("value_for_stimulated_point", 20.0))
        fe = a(spec["firing_events"], np.uint8)
        p.firing_events = _p(fe, C.c_uint8)
        p.firing_rows, p.firing_cols = fe.shape
        p.motor_unit_no = _p(a(spec["motor_unit_no"], np.int32), C.c_int)
        p.stimulation_point_index = _p(a(spec["stimulation_point_index"], np.int32), C.c_int)
        p.call_frequency = _p(a(spec["call_frequency"], np.float64), C.c_double)
        p.repeat_after_first_call = _p(a(spec["repeat_after_first_call"], np.float64), C.c_double)
        p.call_enable_begin = _p(a(spec["call_enable_begin"], np.float64), C.c_double)
        jit = a(spec.get("jitter", np.zeros((p.n_fibers, 0))), np.float64)
        p.n_jitter = jit.shape[1] if jit.ndim == 2 else 0
        p.jitter = _p(jit if jit.size else np.zeros(1), C.c_double)
        p.t_start = float(spec.get("t_start", 0.0))
        p.t_end = float(spec["t_end"])
        p.dt_repeated_call = float(spec.get("dt_repeated_call", spec["dt_splitting"]))
        p.dt_splitting = float(spec["dt_splitting"])
        p.dt_0d = float(spec["dt_0d"])
        p.dt_1d = float(spec["dt_1d"])
        p.n_threads = int(spec.get("n_threads", 1))
        self.n_nodes = int(offsets[-1])
        alg_idx = a(spec.get("algebraic_indices", []), np.int32)
        p.n_algebraics_out = len(alg_idx)
        p.algebraic_indices = _p(alg_idx if len(alg_idx) else np.zeros(1, np.int32), C.c_int)
        self.algebraics = np.zeros((max(len(alg_idx), 1), self.n_nodes))
        p.algebraics_out = _p(self.algebraics, C.c_double)
        tn = a(spec.get("trace_nodes", []), np.int64)
        p.n_trace_nodes = len(tn)
        p.trace_nodes = _p(tn if len(tn) else np.zeros(1, np.int64), C.c_int64)
        cap = int(spec.get("trace_capacity", 0))
        self.trace = np.full((max(cap, 1), max(len(tn), 1)), np.nan)
        p.trace = _p(self.trace, C.c_double)
        p.trace_capacity = cap
        p.only_if_stimulated = int(bool(spec.get("only_if_stimulated", False)))
        nf = p.n_fibers
        # equilibrium skip: statuses of every rank's buffers (all active), counters, padding-lane states
        p.equilibrium = int(bool(spec.get("equilibrium", False)))
        W, R = p.vc_width, p.n_ranks
        lengths = np.diff(offsets)
        n_buf = [int((lengths[r::R].sum() + W - 1) // W) for r in range(R)]
        self.eq_status = np.full(max(sum(n_buf), 1), 2, np.uint8)
        self.eq_counter = np.zeros(R, np.int32)
        ns = model_info(spec["model"])[0]
        self.n_states = ns
        init = model_info(spec["model"])[3]
        self.pad_states = np.tile(init, R * W).astype(np.float64)
        p.eq_status = _p(self.eq_status, C.c_uint8)
        p.eq_counter = _p(self.eq_counter, C.c_int)
        p.pad_states = _p(self.pad_states, C.c_double)
        self.has_been_stimulated = np.zeros(max(nf, 1), np.int32)
        p.has_been_stimulated = _p(self.has_been_stimulated, C.c_int)
        # stimulation log (stimulation_log() returns it), kept across runs
        self.currently_stimulating = np.zeros(max(nf, 1), np.int32)
        p.currently_stimulating = _p(self.currently_stimulating, C.c_int)
        cap = int(spec.get("log_capacity", 0))
        self.log_times = np.zeros(max(cap, 1))
        self.log_fibers = np.zeros(max(cap, 1), np.int32)
        self.log_count = np.zeros(1, np.int64)
        p.log_times = _p(self.log_times, C.c_double)
        p.log_fibers = _p(self.log_fibers, C.c_int)
        p.log_capacity = cap
        p.log_count = _p(self.log_count, C.c_int64) if cap > 0 else None
        self.p = p
        self.last_check_time = np.zeros(nf)
        self.current_jitter = np.zeros(nf)
        self.jitter_index = np.zeros(nf, np.int32)
        lib().oracle_stimulation_init(C.byref(p), _p(self.last_check_time, C.c_double),
                                      _p(self.current_jitter, C.c_double), _p(self.jitter_index, C.c_int))

    def _arr(self, x, dt):
        arr = np.ascontiguousarray(np.asarray(x, dtype=dt))
        if arr.size == 0:
            arr = np.zeros(max(arr.shape[0] if arr.ndim else 1, 1), dtype=dt) if arr.ndim <= 1 else arr
        self.keep.append(arr)
        return arr

    def run(self, states: np.ndarray, t_start: Optional[float] = None, t_end: Optional[float] = None) -> int:
        """Advance the SoA states [s][node] in place; returns the number of split steps."""
        assert states.dtype == np.float64 and states.flags.c_contiguous
        if states.shape != (self.n_states, self.n_nodes):
            raise ValueError(f"oracle run: states must be [{self.n_states}, {self.n_nodes}], got {states.shape}")
        if t_start is not None:
            self.p.t_start = t_start
        if t_end is not None:
            self.p.t_end = t_end
        n = lib().oracle_run(C.byref(self.p), _p(states, C.c_double), _p(self.last_check_time, C.c_double),
                             _p(self.current_jitter, C.c_double), _p(self.jitter_index, C.c_int))
        if n < 0:
            raise RuntimeError("oracle_run failed")
        return int(n)

    def stimulation_log(self):
        """(times, fibers) of the logged stimulation begins, in the order they were recorded (with several
        threads not in time order), and the number of entries that did not fit."""
        n = int(self.log_count[0])
        k = min(n, int(self.p.log_capacity))
        return self.log_times[:k].copy(), self.log_fibers[:k].copy(), n - k

    def vc_clamp_nodes(self):
        nf = self.p.n_fibers
        first = np.zeros(nf, np.int64)
        cnt = np.zeros(nf, np.int32)
        lib().oracle_vc_clamp_nodes(C.byref(self.p), _p(first, C.c_int64), _p(cnt, C.c_int))
        return first, cnt
