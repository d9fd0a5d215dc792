"""Fiber sharding across devices (multi-GPU without a data-path collective).

The reference distributes the fibers of a muscle over MPI ranks; its FastMonodomainSolver then gathers every
fiber onto one rank and solves it there (fast_monodomain_solver_communication.tpp:13-228), so that a fiber is
always solved whole by one process and fibers never exchange data during a solve.  Here a fiber system is
split into shards of whole fibers, one shard per GPU, balanced by the longest-processing-time rule on node
counts (the work of a fiber is proportional to its nodes).  Each shard is an ordinary
:class:`~opendihu_b200.solver.FastMonodomainSolver` on its own device and stream; nothing crosses devices
while they run.  The only exchange is the optional end-of-interval gather of Vm / states into the global node
order (host arrays here, or ``torch.distributed`` gather for one-process-per-GPU jobs).

Results are identical to the unsharded solve: a shard keeps each fiber's geometry, stimulation inputs,
parameters and states, and its junction clamp nodes are those the unsharded layout selects
(:func:`opendihu_b200._native.select_clamp_nodes` on the whole system, mapped to shard-local node indices),
since the "vc" clamp rule depends on how all fibers of a rank are laid out together.
"""
from __future__ import annotations

import ctypes as C
import heapq
import threading
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import _native as N
from . import output
from .solver import (CLAMP_RULES, FastMonodomainSolver, FiberSystem, equilibrium_states, output_writers,
                     piece_end, write_due_output)


def lpt_partition(weights: Sequence[int], n_shards: int) -> List[np.ndarray]:
    """Longest-processing-time assignment: items by decreasing weight (ties by index), each to the shard with
    the least total so far (ties by shard number).  Returns the item indices of every shard in ascending
    order.  Deterministic, so every rank of a distributed job computes the same partition."""
    if n_shards < 1:
        raise ValueError("n_shards must be >= 1")
    w = np.asarray(weights, np.int64)
    order = sorted(range(len(w)), key=lambda i: (-int(w[i]), i))
    heap = [(0, k) for k in range(n_shards)]
    parts: List[List[int]] = [[] for _ in range(n_shards)]
    for i in order:
        load, k = heapq.heappop(heap)
        parts[k].append(i)
        heapq.heappush(heap, (load + int(w[i]), k))
    return [np.asarray(sorted(p), np.int64) for p in parts]


def subset(system: FiberSystem, fibers) -> FiberSystem:
    """The given fibers of a system, as a system of their own (same per-fiber inputs, node order = the given
    fiber order)."""
    fibers = np.asarray(fibers, np.int64)
    off = np.asarray(system.fiber_offsets, np.int64)
    lengths = off[fibers + 1] - off[fibers]
    new_off = np.zeros(len(fibers) + 1, np.int64)
    new_off[1:] = np.cumsum(lengths)
    elem = np.asarray(system.element_lengths)
    elem = np.concatenate([elem[off[f] - f:off[f + 1] - f - 1] for f in fibers]) if len(fibers) else elem[:0]
    nodes = node_index(off, fibers)
    s = system.copy()
    s.fiber_offsets = new_off
    s.element_lengths = elem
    for name in ("prefactor", "motor_unit_no", "stimulation_point_index", "call_frequency",
                 "repeat_after_first_call", "call_enable_begin"):
        setattr(s, name, np.asarray(getattr(system, name))[fibers].copy())
    if system.jitter is not None and np.asarray(system.jitter).size:
        s.jitter = np.asarray(system.jitter)[fibers].copy()
    else:
        s.jitter = np.zeros((len(fibers), 0))
    if system.parameters is not None:
        s.parameters = np.asarray(system.parameters)[:, nodes].copy()
    if system.states is not None:
        s.states = np.asarray(system.states)[:, nodes].copy()
    if len(system.fiber_mesh_names) == system.n_fibers:
        s.fiber_mesh_names = [system.fiber_mesh_names[int(f)] for f in fibers]
    nums = system.fiber_numbers if len(system.fiber_numbers) == system.n_fibers else range(system.n_fibers)
    s.fiber_numbers = [int(nums[int(f)]) for f in fibers]
    # output writers name fibers of the unsharded layout: a shard runs none; the stimulation log file and the
    # equilibrium start belong to the whole system (ShardedSolver writes the one, computes the other once)
    s.output_writers = ()
    s.stimulation_log_filename = ""
    s.initialize_states_to_equilibrium = False
    return s


def node_index(fiber_offsets, fibers) -> np.ndarray:
    """Global node indices of the given fibers, concatenated in the given order."""
    off = np.asarray(fiber_offsets, np.int64)
    fibers = np.asarray(fibers, np.int64)
    if not len(fibers):
        return np.zeros(0, np.int64)
    return np.concatenate([np.arange(off[f], off[f + 1]) for f in fibers])


def global_clamp_nodes(system: FiberSystem):
    """Clamp nodes (first node, count, evaluated per fiber) that the unsharded system selects."""
    return N.select_clamp_nodes(CLAMP_RULES[system.clamp_rule], int(system.vc_width), int(system.n_ranks),
                                system.fiber_offsets, system.stimulation_point_index)


def global_gate_codes(system: FiberSystem) -> np.ndarray:
    """onlyComputeIfHasBeenStimulated codes (attributed fiber * 4 + class per node) of the unsharded system."""
    return N.select_gate_codes(CLAMP_RULES[system.clamp_rule], int(system.vc_width), int(system.n_ranks),
                               system.fiber_offsets, system.stimulation_point_index)


def shard_gate_codes(system: FiberSystem, fibers, codes) -> np.ndarray:
    """The global codes of the shard's nodes with the attributed fibers renumbered shard-locally; a node
    attributed to a fiber of another shard (possible with the vc rule and uneven lengths) cannot be gated
    without an exchange, so that raises."""
    fibers = np.asarray(fibers, np.int64)
    local = np.full(len(system.fiber_offsets) - 1, -1, np.int64)
    local[fibers] = np.arange(len(fibers))
    c = np.asarray(codes, np.int64)[node_index(system.fiber_offsets, fibers)]
    att = local[c >> 2]
    if np.any(att < 0):
        raise ValueError("onlyComputeIfHasBeenStimulated: a point buffer of this shard is attributed to a fiber of "
                         "another shard (vc rule with uneven fiber lengths); use the centre rule or one shard")
    return (att * 4 + (c & 3)).astype(np.int32)


def shard_clamp_nodes(system: FiberSystem, fibers, clamp):
    """The global clamp selection restricted to the given fibers, as shard-local node indices."""
    first, cnt, ev = clamp
    fibers = np.asarray(fibers, np.int64)
    off = np.asarray(system.fiber_offsets, np.int64)
    lengths = off[fibers + 1] - off[fibers]
    local_off = np.concatenate([[0], np.cumsum(lengths)[:-1]]).astype(np.int64)
    f_first = first[fibers]
    local_first = np.where(f_first >= 0, f_first - off[fibers] + local_off, -1).astype(np.int64)
    return local_first, cnt[fibers].astype(np.int32), ev[fibers].astype(np.uint8)


class ShardedSolver:
    """One fiber system solved as LPT shards on several devices (or several shards on one device).

    Mirrors the operator API of :class:`FastMonodomainSolver` (``initialize``, ``setTimeSpan``,
    ``advanceTimeSpan``, ``run``, ``states``, ``vm``, ``set_states``, ``parameters``, checkpoints, adjoint) on
    the global node order.  Each shard's calls run on their own host thread so that devices advance
    concurrently (the C ABI releases the interpreter lock for the length of every call)."""

    def __init__(self, system: FiberSystem, devices: Sequence[int] = (0,), n_shards: Optional[int] = None,
                 **solver_kw):
        self.system = system
        devices = list(devices)
        n = int(n_shards or len(devices))
        if n < 1 or not devices:
            raise ValueError("need at least one shard and one device")
        lengths = np.diff(np.asarray(system.fiber_offsets, np.int64))
        self.fibers = lpt_partition(lengths, n)
        self.devices = [devices[k % len(devices)] for k in range(n)]
        clamp = global_clamp_nodes(system)
        gate = global_gate_codes(system) if system.only_compute_if_has_been_stimulated else None
        self.nodes = [node_index(system.fiber_offsets, f) for f in self.fibers]
        self.shards: List[Optional[FastMonodomainSolver]] = []
        for fib, dev in zip(self.fibers, self.devices):
            if not len(fib):
                self.shards.append(None)
                continue
            sub = subset(system, fib)
            sv = FastMonodomainSolver(sub, device=dev, **solver_kw)
            sv.clamp_override = shard_clamp_nodes(system, fib, clamp)
            if gate is not None:
                sv.gate_override = shard_gate_codes(system, fib, gate)
            self.shards.append(sv)
        self._start = system.start_time
        self._end = system.end_time
        self._log_on = False
        self._writers = None
        self._current_time = system.start_time
        self._piece_steps = 0
        #: result of the "initializeStatesToEquilibrium" search, when the settings ask for it
        self.equilibrium = None

    # -- parallel dispatch ------------------------------------------------------------------------
    def _each(self, fn):
        """fn(shard_index, solver) on every non-empty shard, one host thread per shard; re-raises the first
        error after all threads joined."""
        results: Dict[int, object] = {}
        errors: List[BaseException] = []

        def work(k, sv):
            try:
                results[k] = fn(k, sv)
            except BaseException as e:  # noqa: BLE001 - re-raised below
                errors.append(e)

        live = [(k, sv) for k, sv in enumerate(self.shards) if sv is not None]
        if len(live) == 1:
            work(*live[0])
        else:
            th = [threading.Thread(target=work, args=(k, sv)) for k, sv in live]
            for t in th:
                t.start()
            for t in th:
                t.join()
        if errors:
            raise errors[0]
        return results

    # -- lifecycle and the operator API ----------------------------------------------------------
    def initialize(self):
        s = self.system
        if s.initialize_states_to_equilibrium and self.equilibrium is None:
            # one search for the whole system (the first node's states and parameters), as unsharded
            self.equilibrium = equilibrium_states(s, self.devices[0])
            s.states = np.repeat(self.equilibrium["states"][:, None], s.n_nodes, axis=1)
            for k, sv in enumerate(self.shards):
                if sv is not None:
                    sv.system.states = np.ascontiguousarray(s.states[:, self.nodes[k]])
        self._each(lambda k, sv: sv.initialize())
        if s.stimulation_log_filename and not self._log_on:
            self._log_on = True
            self._each(lambda k, sv: sv.enable_stimulation_log())

    def stimulation_log(self) -> Dict[str, np.ndarray]:
        """The shards' stimulation logs merged, fibers by their numbers in the whole system, in time order."""
        r = self._each(lambda k, sv: sv.stimulation_log())
        t = np.concatenate([d["time"] for d in r.values()]) if r else np.zeros(0)
        f = np.concatenate([d["fiber"] for d in r.values()]) if r else np.zeros(0, np.int64)
        m = np.concatenate([d["motorUnit"] for d in r.values()]) if r else np.zeros(0, np.int64)
        order = np.lexsort((f, t))
        return {"time": t[order], "fiber": f[order], "motorUnit": m[order]}

    def writeStimulationLog(self, filename: Optional[str] = None) -> str:
        name = filename or self.system.stimulation_log_filename
        if not name:
            raise ValueError("writeStimulationLog: no file name (settings have no stimulationLogFilename)")
        d = self.stimulation_log()
        output.write_stimulation_log(name, d["time"], d["fiber"], d["motorUnit"])
        return name

    def close(self):
        try:
            if self.system.stimulation_log_filename and self._log_on and any(sv is not None and sv.initialized
                                                                             for sv in self.shards):
                self.writeStimulationLog()
        finally:
            for sv in self.shards:
                if sv is not None:
                    sv.close()

    def __enter__(self):
        self.initialize()
        return self

    def __exit__(self, *exc):
        self.close()

    def setTimeSpan(self, start_time: float, end_time: float):
        self._start, self._end = float(start_time), float(end_time)
        for sv in self.shards:
            if sv is not None:
                sv.setTimeSpan(start_time, end_time)

    def startTime(self) -> float:
        return self._start

    def endTime(self) -> float:
        return self._end

    def advanceTimeSpan(self, withOutputWritersEnabled: bool = True):
        """Every shard advances over [startTime, endTime].  With the settings' output writers (enabled) the shards
        stop together after each RepeatedCall piece whose call writes, and the writers get the whole system's
        fibers (as FastMonodomainSolver.advanceTimeSpan, fast_monodomain_solver_compute.tpp:35-44)."""
        self.initialize()
        live = [sv for sv in self.shards if sv is not None]
        if not live:
            return
        writers = self._output_writers() if withOutputWritersEnabled else []
        n, steps = self._plan(live[0])
        if not writers:
            self._each(lambda k, sv: sv.advanceTimeSpan(withOutputWritersEnabled))
        else:
            self._each(lambda k, sv: sv._prepare_advance())
            done = 0
            for k in range(n):
                t = piece_end(self._start, self._end, k, n)
                due = [(w, name) for w in writers for name in [w.prepare(0, t, int(steps[k]))] if name]
                self._current_time, self._piece_steps = t, int(steps[k])
                if due:
                    k0, k1 = done, k + 1
                    self._each(lambda j, sv: sv._advance_pieces(k0, k1))
                    done = k1
                    write_due_output(self, due, t)
            if done < n:
                k0 = done
                self._each(lambda j, sv: sv._advance_pieces(k0, n))
        self._current_time = piece_end(self._start, self._end, n - 1, n)
        self._piece_steps = int(steps[n - 1])

    def _plan(self, sv):
        """The RepeatedCall pieces of the span and their split steps (every shard plans alike)."""
        nn = C.c_int64()
        N.check(N.lib().fdm_repeated_call_plan(sv._h, self._start, self._end, C.byref(nn), None), sv._h)
        steps = np.zeros(max(nn.value, 1), np.int32)
        if self.system.output_writers:
            N.check(N.lib().fdm_repeated_call_plan(sv._h, self._start, self._end, C.byref(nn),
                                                   N.ptr(steps, C.c_int)), sv._h)
        return nn.value, steps

    def _output_writers(self):
        if self._writers is None:
            self._writers = output_writers(self.system)
        return self._writers

    def callOutputWriter(self, timeStepNo: int, currentTime: float, callCountIncrement: int = 1):
        """FastMonodomainSolver.callOutputWriter over the whole system."""
        self.initialize()
        if int(timeStepNo) % int(callCountIncrement) != 0:
            return
        due = [(w, name) for w in self._output_writers()
               for name in [w.prepare(0, self._current_time, self._piece_steps)] if name]
        if due:
            write_due_output(self, due, self._current_time)

    def compute_state_information(self) -> np.ndarray:
        r = self._each(lambda k, sv: sv.compute_state_information()[None, :])
        return self._gather_rows(r, 1)[0]

    def run(self):
        self.initialize()
        self.advanceTimeSpan()

    def saveFiberDataCheckpoint(self):
        self._each(lambda k, sv: sv.saveFiberDataCheckpoint())

    def restoreFiberDataCheckpoint(self):
        self._each(lambda k, sv: sv.restoreFiberDataCheckpoint())

    def rewind(self):
        self._each(lambda k, sv: sv.rewind())

    # -- gathers into the global node order -----------------------------------------------------
    def _gather_rows(self, per_shard: Dict[int, np.ndarray], n_rows: int) -> np.ndarray:
        out = np.zeros((n_rows, self.system.n_nodes))
        for k, a in per_shard.items():
            out[:, self.nodes[k]] = a
        return out

    def states(self) -> np.ndarray:
        r = self._each(lambda k, sv: sv.states())
        return self._gather_rows(r, next(iter(r.values())).shape[0])

    def vm(self) -> np.ndarray:
        r = self._each(lambda k, sv: sv.vm()[None, :])
        return self._gather_rows(r, 1)[0]

    def algebraics(self) -> np.ndarray:
        r = self._each(lambda k, sv: sv.algebraics())
        return self._gather_rows(r, len(self.system.algebraics_for_transfer))

    def parameters(self) -> np.ndarray:
        r = self._each(lambda k, sv: sv.parameters())
        return self._gather_rows(r, next(iter(r.values())).shape[0])

    def set_states(self, states: np.ndarray):
        states = np.asarray(states, np.float64)
        self._each(lambda k, sv: sv.set_states(states[:, self.nodes[k]]))

    def set_parameters(self, params: np.ndarray):
        params = np.asarray(params, np.float64)
        self._each(lambda k, sv: sv.set_parameters(params[:, self.nodes[k]]))

    def set_prefactor(self, prefactor: np.ndarray):
        prefactor = np.asarray(prefactor, np.float64)
        self._each(lambda k, sv: sv.set_prefactor(prefactor[self.fibers[k]]))

    def split_steps(self) -> int:
        return max(sv.split_steps() for sv in self.shards if sv is not None)

    def timing(self) -> List[Dict[str, float]]:
        return [sv.timing() if sv is not None else None for sv in self.shards]

    # -- adjoint: every shard differentiates its own fibers -------------------------------------
    def adjoint_forward(self, t_start: float, t_end: float, checkpoint_every: int, sensor_nodes) -> np.ndarray:
        """Checkpointed forward of every shard; returns the trace [steps, sensors] in the given sensor order."""
        sensor_nodes = np.asarray(sensor_nodes, np.int64)
        owner = np.full(self.system.n_nodes, -1, np.int64)
        local = np.zeros(self.system.n_nodes, np.int64)
        for k, nodes in enumerate(self.nodes):
            owner[nodes] = k
            local[nodes] = np.arange(len(nodes))
        self._sensor_split = {k: np.nonzero(owner[sensor_nodes] == k)[0] for k in range(len(self.shards))}
        r = self._each(lambda k, sv: sv.adjoint_forward(t_start, t_end, checkpoint_every,
                                                        local[sensor_nodes[self._sensor_split[k]]]))
        steps = max(a.shape[0] for a in r.values())
        out = np.zeros((steps, len(sensor_nodes)))
        for k, a in r.items():
            out[:a.shape[0], self._sensor_split[k]] = a
        return out

    def adjoint(self, t_start: float, t_end: float, checkpoint_every: int, sensor_nodes,
                loss_grad: Callable[[np.ndarray, np.ndarray], np.ndarray]):
        """The adjoint one shard after the other, each shard's checkpoints and replay buffers freed before the
        next starts (device memory for one shard's adjoint at a time, see plan_adjoint).  The loss must be a sum
        over sensors: loss_grad(trace, sensors) gets a shard's trace [steps, k] and the positions of its k
        sensors in sensor_nodes and returns dL/dtrace for them.  Returns (trace [steps, sensors], gradients)."""
        sensor_nodes = np.asarray(sensor_nodes, np.int64)
        owner = np.full(self.system.n_nodes, -1, np.int64)
        local = np.zeros(self.system.n_nodes, np.int64)
        for k, nodes in enumerate(self.nodes):
            owner[nodes] = k
            local[nodes] = np.arange(len(nodes))
        traces, grads = {}, {}
        #: device time (CUDA events) of the last adjoint: checkpointed forwards and backward sweeps of all shards
        self.adjoint_device_ms = {"checkpointed_forward_ms": 0.0, "backward_ms": 0.0}
        for k, sv in enumerate(self.shards):
            if sv is None:
                continue
            cols = np.nonzero(owner[sensor_nodes] == k)[0]
            sv.initialize()
            sv.reset_timing()
            tr = sv.adjoint_forward(t_start, t_end, checkpoint_every, local[sensor_nodes[cols]])
            self.adjoint_device_ms["checkpointed_forward_ms"] += sv.timing()["advance_ms"]
            grads[k] = sv.adjoint_backward(loss_grad(tr, cols))
            self.adjoint_device_ms["backward_ms"] += sv.adjoint_timing_ms()
            sv.adjoint_release()
            traces[k] = (cols, tr)
        steps = max(tr.shape[0] for _, tr in traces.values())
        out = np.zeros((steps, len(sensor_nodes)))
        for cols, tr in traces.values():
            out[:tr.shape[0], cols] = tr
        return out, self._merge_gradients(grads)

    def _merge_gradients(self, r: Dict[int, Dict[str, np.ndarray]]) -> Dict[str, np.ndarray]:
        nf, nn = self.system.n_fibers, self.system.n_nodes
        any_r = next(iter(r.values()))
        g = {"prefactor": np.zeros(nf), "parameters": np.zeros((any_r["parameters"].shape[0], nn)),
             "states0": np.zeros((any_r["states0"].shape[0], nn))}
        for k, a in r.items():
            g["prefactor"][self.fibers[k]] = a["prefactor"]
            g["parameters"][:, self.nodes[k]] = a["parameters"]
            g["states0"][:, self.nodes[k]] = a["states0"]
        return g

    def adjoint_backward(self, trace_grad: np.ndarray) -> Dict[str, np.ndarray]:
        tg = np.asarray(trace_grad, np.float64)
        r = self._each(lambda k, sv: sv.adjoint_backward(tg[:, self._sensor_split[k]]))
        return self._merge_gradients(r)


def adjoint_bytes_per_node(model: str, n_substeps: int, n_steps: int, checkpoint_every: int) -> int:
    """Device bytes per node the FP64 adjoint holds (fdm_adjoint_forward / fdm_adjoint_backward): one
    checkpoint of the states per segment, two replay buffers of a segment's Heun substep states (the replay of
    one segment overlaps the reverse sweep of the next) with Vm before each diffusion solve, and the adjoint
    variables; n_substeps = Heun substeps per half step."""
    from .solver import model_sizes
    ns, _, npar = model_sizes(model)[:3]
    kc = max(1, min(int(checkpoint_every), int(n_steps)))
    segments = -(-int(n_steps) // kc)
    checkpoints = segments * ns * 8
    replay = 2 * kc * (2 * n_substeps * ns + 1) * 8
    adjoint = (ns + max(npar, 1) + 3) * 8
    return checkpoints + replay + adjoint


def plan_adjoint(system: FiberSystem, t_start: float, t_end: float, budget_bytes: float) -> Dict[str, int]:
    """Checkpoint interval and number of sequential fiber shards for an FP64 adjoint over [t_start, t_end] that
    fits budget_bytes of device memory: the interval minimising the per-node memory (checkpoints ~ S/k against
    replay ~ k, so k ~ sqrt(S / (4 n0))), then as many LPT shards as the largest shard needs to fit."""
    import math
    dt = system.dt_splitting
    n_steps = max(1, int(math.ceil((t_end - t_start) / dt - 0.1)))
    n0 = max(1, int(math.ceil(0.5 * dt / system.dt_0d - 0.1)))
    best = None
    k0 = max(1, int(round(math.sqrt(n_steps / (4.0 * n0)))))
    for k in sorted({max(1, k0 // 2), k0, k0 + 1, 2 * k0, 1}):
        b = adjoint_bytes_per_node(system.model, n0, n_steps, k)
        if best is None or b < best[1]:
            best = (k, b)
    k, per_node = best
    lengths = np.diff(np.asarray(system.fiber_offsets, np.int64))
    n_shards = 1
    while True:
        parts = lpt_partition(lengths, n_shards)
        largest = max(int(lengths[p].sum()) for p in parts if len(p)) if len(lengths) else 0
        if largest * per_node <= budget_bytes or n_shards >= max(len(lengths), 1):
            break
        n_shards += 1
    if largest * per_node > budget_bytes:
        raise ValueError(f"one fiber alone needs {largest * per_node / 1e9:.1f} GB for the adjoint")
    return {"checkpoint_every": k, "n_shards": n_shards, "bytes_per_node": per_node, "n_steps": n_steps,
            "largest_shard_nodes": largest}


def rank_shard(system: FiberSystem, rank: int, world: int):
    """The shard of one rank of a one-process-per-GPU job: (fiber indices, shard system, clamp override)."""
    fibers = lpt_partition(np.diff(np.asarray(system.fiber_offsets, np.int64)), world)[rank]
    return fibers, subset(system, fibers), shard_clamp_nodes(system, fibers, global_clamp_nodes(system))


def gather_to_root(pg, system: FiberSystem, fibers, local_rows: np.ndarray, root: int = 0):
    """End-of-interval gather of per-rank rows [rows, shard nodes] into the global node order on ``root``
    (``torch.distributed``; returns None on the other ranks).  Object gather: an end-of-interval copy, not
    part of the time-stepping."""
    import torch.distributed as dist
    rank = dist.get_rank(pg)
    world = dist.get_world_size(pg)
    payload = (np.asarray(fibers, np.int64), np.asarray(local_rows))
    got = [None] * world if rank == root else None
    dist.gather_object(payload, got, dst=root, group=pg)
    if rank != root:
        return None
    out = np.zeros((payload[1].shape[0], system.n_nodes))
    for fib, rows in got:
        out[:, node_index(system.fiber_offsets, fib)] = rows
    return out
