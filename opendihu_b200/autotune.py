"""Autotuner of the fused kernel's launch shape.

The fused kernel packs whole fibers into bins of T*M nodes (T threads per CTA, M nodes per thread, so the
number of fibers per CTA follows from the fiber lengths) and runs K Strang steps per launch; in cluster mode
it spreads each fiber over C CTAs of a thread-block cluster.  The best (T, M, C) depends on the model's
register footprint and on the length distribution (bin fill, waves on 148 SMs: 169 fibers in 169 bins run
in two waves, spread over clusters they fill the GPU evenly); K trades launch overhead against
stimulation-schedule memory.  The tuner times every built shape that holds the longest fiber (cluster shapes
with 2..8 CTAs per fiber where the model and options allow them) on the actual workload for a few Strang
steps (device time of the kernel launches, CUDA events) and then a few K values for the winner.  Results are cached per workload signature
in memory and, if FDM_AUTOTUNE_CACHE names a file, in that JSON file.
"""
from __future__ import annotations

import hashlib
import json
import os
from typing import Dict, Optional, Sequence

import numpy as np

from . import _native as N

_MEMO: Dict[str, dict] = {}


def signature(system, precision: str) -> str:
    lengths = np.diff(np.asarray(system.fiber_offsets))
    hist = np.histogram(lengths, bins=16, range=(0, int(lengths.max()) + 1))[0]
    desc = [system.model, precision, system.diffusion_scheme, bool(system.approximate_exponential_function),
            bool(getattr(system, "only_compute_if_has_been_stimulated", False)), int(lengths.max()),
            int(lengths.sum()), hist.tolist(), "cluster"]
    return hashlib.sha1(json.dumps(desc).encode()).hexdigest()[:16]


def _load_cache() -> Dict[str, dict]:
    path = os.environ.get("FDM_AUTOTUNE_CACHE")
    if path and os.path.exists(path):
        try:
            return json.load(open(path))
        except (OSError, ValueError):
            return {}
    return {}


def _store_cache(key: str, value: dict):
    path = os.environ.get("FDM_AUTOTUNE_CACHE")
    if not path:
        return
    data = _load_cache()
    data[key] = value
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1)
    os.replace(tmp, path)


def _time_shape(system, precision, threads, m, k, n_steps, device, cluster_size: int = 1) -> float:
    """Seconds of device time per Strang step (all GPU work of the advance: schedule + fused kernels)."""
    from .solver import FastMonodomainSolver
    s = system.copy()
    dt = s.dt_splitting
    with FastMonodomainSolver(s, method="fused", precision=precision, threads_per_block=threads,
                              nodes_per_thread=m, steps_per_launch=k, profile=True, device=device,
                              check_nan=False, cluster_size=cluster_size) as slv:
        slv.setTimeSpan(s.start_time, s.start_time + dt * min(k, n_steps))
        slv.advanceTimeSpan()  # warm-up (module load, factorization)
        slv.reset_timing()
        t0 = s.start_time + dt * min(k, n_steps)
        slv.setTimeSpan(t0, t0 + dt * n_steps)
        slv.advanceTimeSpan()
        tm = slv.timing()
    return tm["advance_ms"] / 1e3 / n_steps


def _time_split(system, precision, k, n_steps, device) -> float:
    """Seconds of device time per Strang step of the split method (window launches replayed as CUDA graphs)."""
    from .solver import FastMonodomainSolver
    s = system.copy()
    dt = s.dt_splitting
    with FastMonodomainSolver(s, method="split", precision=precision, steps_per_launch=k, device=device,
                              check_nan=False) as slv:
        slv.setTimeSpan(s.start_time, s.start_time + dt * min(k, n_steps))
        slv.advanceTimeSpan()
        slv.reset_timing()
        t0 = s.start_time + dt * min(k, n_steps)
        slv.setTimeSpan(t0, t0 + dt * n_steps)
        slv.advanceTimeSpan()
        tm = slv.timing()
    return tm["advance_ms"] / 1e3 / n_steps


def _fused_built(system, precision, device) -> bool:
    """Whether the library builds the fused kernel for the model (fdm_create refuses it otherwise; nothing is
    allocated before that check)."""
    import ctypes as C
    cfg = N.default_config()
    cfg.model = N.MODEL_IDS[system.model]
    cfg.method = 1
    cfg.reaction_precision = 0 if precision == "fp64" else 1
    cfg.device = int(device)
    h = C.c_void_p()
    rc = N.lib().fdm_create(C.byref(cfg), C.byref(h))
    if rc == N.FDM_OK:
        N.lib().fdm_destroy(h)
        return True
    if rc == N.FDM_ERR_UNSUPPORTED:
        return False
    N.check(rc)
    return True


def autotune(system, precision: str = "fp32", n_steps: int = 20, device: int = 0,
             steps_per_launch: Sequence[int] = (50, 100, 200), use_cache: bool = True,
             include_split: bool = False) -> dict:
    """Return {"method", "threads", "nodes_per_thread", "cluster_size", "steps_per_launch", "s_per_step",
    "trials"} for the workload (cluster_size 1: bins of whole fibers).  With include_split the split method (a
    reaction launch per half step and a diffusion launch per step, as CUDA graphs) competes too: with few
    nodes its one thread per node can outrun the fused kernel's shapes."""
    if include_split and getattr(system, "skip_close_to_equilibrium", False):
        return {"method": "split", "threads": 0, "nodes_per_thread": 0, "cluster_size": 1, "steps_per_launch": 0,
                "s_per_step": None, "trials": [], "reason": "the equilibrium skip runs on the split method"}
    if include_split and not _fused_built(system, precision, device):
        return {"method": "split", "threads": 0, "nodes_per_thread": 0, "cluster_size": 1, "steps_per_launch": 0,
                "s_per_step": None, "trials": [], "reason": "no fused kernel is built for this model"}
    key = signature(system, precision) + ("+split" if include_split else "")
    if use_cache:
        if key in _MEMO:
            return _MEMO[key]
        cached = _load_cache().get(key)
        if cached:
            _MEMO[key] = cached
            return cached
    max_len = int(np.diff(np.asarray(system.fiber_offsets)).max())
    shapes = [(t, m, 1) for t, m in N.fused_shapes() if t * m >= max_len]
    if (system.model == "hodgkin_huxley_1952" and not system.approximate_exponential_function
            and not getattr(system, "only_compute_if_has_been_stimulated", False)):
        for t, m in N.fused_shapes(cluster=True):
            c = -(-max_len // (t * m))
            if 2 <= c <= 8:
                shapes.append((t, m, c))
    if not shapes and not include_split:
        raise N.FdmError(N.FDM_ERR_UNSUPPORTED, f"no fused shape holds a fiber of {max_len} nodes")
    trials = []
    if include_split:
        trials.append({"method": "split", "threads": 0, "nodes_per_thread": 0, "cluster_size": 1,
                       "steps_per_launch": 100, "s_per_step": _time_split(system, precision, 100, max(n_steps, 100),
                                                                         device)})
        if not shapes:
            result = dict(trials[0])
            result["trials"] = trials
            _MEMO[key] = result
            if use_cache:
                _store_cache(key, result)
            return result
    k0 = 100
    for t, m, c in shapes:
        try:
            sec = _time_shape(system, precision, t, m, min(k0, n_steps), n_steps, device, c)
        except N.FdmError as e:
            if e.code != N.FDM_ERR_UNSUPPORTED:
                raise
            continue    # a combination the library does not build (a model without a fused kernel)
        trials.append({"method": "fused", "threads": t, "nodes_per_thread": m, "cluster_size": c,
                       "steps_per_launch": min(k0, n_steps), "s_per_step": sec})
    if not trials:
        raise N.FdmError(N.FDM_ERR_UNSUPPORTED, "no fused kernel is built for this workload")
    best = min(trials, key=lambda r: r["s_per_step"])
    if best["method"] == "split":
        result = dict(best)
        result["trials"] = trials
        _MEMO[key] = result
        if use_cache:
            _store_cache(key, result)
        return result
    # window length for the winner, over a span of a few windows
    k_trials = []
    for k in steps_per_launch:
        span = max(n_steps, 2 * k)
        k_trials.append({"method": "fused", "threads": best["threads"], "nodes_per_thread": best["nodes_per_thread"],
                         "cluster_size": best["cluster_size"], "steps_per_launch": k,
                         "s_per_step": _time_shape(system, precision, best["threads"], best["nodes_per_thread"], k,
                                                   span, device, best["cluster_size"])})
    best_k = min(k_trials, key=lambda r: r["s_per_step"])
    result = dict(best_k)
    result["trials"] = trials + k_trials
    _MEMO[key] = result
    if use_cache:
        _store_cache(key, result)
    return result
