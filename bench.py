#!/usr/bin/env python
"""Benchmark of the fiber monodomain hot path: node-steps/s of the FP32-reaction fused solver on the
batched Hodgkin-Huxley workload (4096 fibers of 500-2500 nodes, Crank-Nicolson), next to the FP64
split ("plain") solver, with accuracy against the CPU oracle and the oracle's CPU throughput.

One step = one advance of 1 ms of simulated time (1000 Strang steps) over the whole batch.
Multi-GPU (torchrun): every rank solves its own batch (seed = rank): fibers are independent, there
is no data-path collective, scaling is weak; the timed region is bracketed by barriers and the
reported time is the maximum over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
METRIC = "node-steps/s, FP32 batched vs FP64 plain at <=0.1 mV; adjoint/forward time"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--step-ms", type=float, default=1.0, help="simulated ms per step")
    p.add_argument("--fibers", type=int, default=4096)
    p.add_argument("--skip-fp64", action="store_true")
    p.add_argument("--skip-accuracy", action="store_true")
    p.add_argument("--threads", type=int, default=0, help="fused CTA threads (0 = default)")
    p.add_argument("--nodes-per-thread", type=int, default=0)
    p.add_argument("--steps-per-launch", type=int, default=0)
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--skip-adjoint", action="store_true")
    p.add_argument("--adjoint-ms", type=float, default=20.0, help="simulated span of the adjoint measurement")
    p.add_argument("--skip-emg", action="store_true")
    p.add_argument("--only", choices=["emg", "emg-cg", "shorten", "plain", "adjoint", "c2-accuracy", "c5"],
                   help="print one side measurement alone (profiling runs)")
    p.add_argument("--accuracy-ms", type=float, default=100.0, help="span of the batch accuracy comparison")
    p.add_argument("--skip-shorten", action="store_true")
    p.add_argument("--skip-c5", action="store_true")
    p.add_argument("--plain-legs", default="", help="comma-separated legs of --only plain (default: all)")
    p.add_argument("--c5-ms", type=float, default=0.5, help="simulated span of the Shorten-at-scale run")
    p.add_argument("--c5-adjoint-steps", type=int, default=4, help="Strang steps of the Shorten-at-scale adjoint")
    p.add_argument("--shorten-ms", type=float, default=0.02, help="simulated span of the Shorten timing (full grid)")
    p.add_argument("--shorten-accuracy-ms", type=float, default=5.0,
                   help="simulated span of the Shorten FP32-vs-FP64 comparison (16-fiber sample)")
    p.add_argument("--emg-cg-mesh", default="97,97,297", help="3D nodes of the CG-iteration measurement")
    p.add_argument("--emg-cg-iterations", type=int, default=160)
    return p.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    if os.path.exists(MEASURED_PEAKS):
        d = json.load(open(MEASURED_PEAKS))
        return d.get("hbm_gbs", FALLBACK_HBM_GBS), d.get("sm_max_mhz", 1965.0), "measured"
    return FALLBACK_HBM_GBS, 1965.0, "fallback"


def hh_ops():
    meta = json.load(open(os.path.join(ROOT, "opendihu_b200/csrc/generated/hodgkin_huxley_1952_anone_c2_3_4.json")))
    return meta["operations_per_rhs"]


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def allmax(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(system, sample_fibers: int, sample_ms: float, threads: int):
    """Oracle (FP64 restatement of the reference's CPU path) on a bounded sample of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers as H
    from opendihu_b200 import workloads as WL
    sub = WL.subset(system, np.arange(sample_fibers))
    sub.end_time = sub.start_time + sample_ms
    H.complete(sub)
    t0 = time.perf_counter()
    st, _, tr, n = H.run_oracle(sub.copy(), n_threads=threads)
    dt = time.perf_counter() - t0
    return sub, st, n, sub.n_nodes * n / dt, dt


def adjoint_measurement(device: int, span_ms: float) -> dict:
    """Differentiation configuration: adjoint gradient cost relative to one FP64 forward solve (256 HH fibers x
    1481 nodes, per-fiber sigma, g_Na, g_K; 32 sensors per fiber; checkpoint every 100 Strang steps)."""
    from opendihu_b200 import adjoint as ADJ
    from opendihu_b200 import solver as S
    from opendihu_b200 import workloads as WL
    dsys, sigma, s_na, s_k, sensors = WL.differentiation_hh(end_time=span_ms, seed=1)
    _, sigma2, s_na2, s_k2, _ = WL.differentiation_hh(end_time=span_ms, seed=2)
    eng = ADJ.AdjointEngine(dsys, sensors, checkpoint_every=100, device=device)
    target = eng.forward(sigma2 / (WL.AM * WL.CM), WL.hh_parameters(dsys, s_na2, s_k2))
    eng.solver.reset_timing()
    trace = eng.forward(dsys.prefactor, dsys.parameters)
    fwd_ck_ms = eng.solver.timing()["advance_ms"]
    loss = float(((trace - target) ** 2).sum())
    g = eng.backward(2.0 * (trace - target))
    bwd_ms = eng.solver.adjoint_timing_ms()
    eng.close()
    with S.FastMonodomainSolver(dsys.copy(), method="split", precision="fp64", device=device) as fw:
        fw.advanceTimeSpan()
        fw.reset_timing()
        fw.rewind()
        fw.set_states(np.repeat(S.model_sizes(dsys.model)[3][:, None], dsys.n_nodes, axis=1))
        fw.advanceTimeSpan()
        plain_fwd_ms = fw.timing()["advance_ms"]
    lengths = np.diff(dsys.fiber_offsets)
    fiber_of = np.repeat(np.arange(dsys.n_fibers), lengths)
    g_na = np.bincount(fiber_of, g["parameters"][1] * 120.0, minlength=dsys.n_fibers)
    return {"workload": "256 HH fibers x 1481 nodes, %g ms, 32 sensors/fiber, checkpoint every 100 steps, "
                        "768 parameters (sigma, g_Na scale, g_K scale per fiber)" % span_ms,
            "forward_ms": plain_fwd_ms, "checkpointed_forward_ms": fwd_ck_ms, "backward_ms": bwd_ms,
            "adjoint_over_forward": (fwd_ck_ms + bwd_ms) / plain_fwd_ms,
            "backward_over_forward": bwd_ms / plain_fwd_ms, "loss": loss,
            "grad_norm_sigma": float(np.linalg.norm(g["prefactor"] / (WL.AM * WL.CM))),
            "grad_norm_gna_scale": float(np.linalg.norm(g_na))}


def plain_measurement(device: int, legs=None) -> dict:
    """The plain-method configuration (16 HH fibers x 1481 nodes, implicit Euler, 10 ms): the FP64 split path
    with CUDA graphs and the fused kernel (cluster mode: few fibers) in FP64 and FP32, 9 ms after 1 ms warm-up."""
    from opendihu_b200 import solver as S
    from opendihu_b200 import workloads as WL
    c1 = WL.plain_hh(end_time=10.0)
    out = {"workload": "16 HH fibers x 1481 nodes, implicit Euler, 10 ms"}
    for name, method, prec in (("fp64_split", "split", "fp64"), ("fp64_fused", "fused", "fp64"),
                               ("fp32_fused", "fused", "fp32"), ("fp64_auto", "auto", "fp64"),
                               ("fp32_auto", "auto", "fp32")):
        if legs and name not in legs:
            continue
        with S.FastMonodomainSolver(c1.copy(), method=method, precision=prec, device=device) as sv:
            sv.setTimeSpan(0.0, 1.0)
            sv.advanceTimeSpan()
            sv.reset_timing()
            sv.setTimeSpan(1.0, 10.0)
            sv.advanceTimeSpan()
            ms = sv.timing()["advance_ms"]
            if method == "fused" and prec == "fp64":
                # few fibers: each fiber spread over the CTAs of a thread-block cluster
                out["fused_layout"] = sv.fused_layout()
            if method == "auto":
                out[name + "_choice"] = {k: sv.tuning.get(k) for k in ("method", "threads", "nodes_per_thread",
                                                                       "cluster_size", "steps_per_launch")}
        out[name] = c1.n_nodes * 9000 / (ms / 1e3)
    return out


def shorten_measurement(device: int, span_ms: float, accuracy_ms: float = 5.0):
    """The Shorten 2007 configuration (56 states; 1369 fibers x 1481 nodes = 2.03M nodes, dt0D 1e-5, dt_split
    5e-4, seeded per-MU firing): FP64 plain (split) against the FP32-reaction path, timed on the full grid over
    a bounded span (the 50 ms of the configuration take minutes; node-steps/s does not depend on the span), and
    compared on a 16-fiber sample of the grid (fibers whose motor unit fires at t = 0, so the span holds action
    potentials) over accuracy_ms: Vm of all nodes and activation steps at 32 nodes per fiber."""
    from opendihu_b200 import accuracy as ACC
    from opendihu_b200 import solver as S
    from opendihu_b200 import workloads as WL
    system = WL.shorten_grid(end_time=span_ms + 0.01)
    out = {"workload": "Shorten 2007, 1369 fibers x 1481 nodes (%d nodes), dt0D 1e-5, dt_split 5e-4 (25 Heun "
                       "substeps per half step), %.3f ms timed after 0.01 ms warm-up" % (system.n_nodes, span_ms)}
    for name, prec in (("fp64_plain", "fp64"), ("fp32_reaction", "fp32")):
        with S.FastMonodomainSolver(system.copy(), method="split", precision=prec, device=device) as sv:
            sv.setTimeSpan(0.0, 0.01)
            sv.advanceTimeSpan()
            sv.reset_timing()
            n0 = sv.split_steps()
            sv.setTimeSpan(0.01, 0.01 + span_ms)
            sv.advanceTimeSpan()
            ms = sv.timing()["advance_ms"]
            steps = sv.split_steps() - n0
        out[name] = {"node_steps_per_s": system.n_nodes * steps / (ms / 1e3), "ms": ms, "strang_steps": steps}
    out["speedup_fp32_over_fp64"] = out["fp32_reaction"]["node_steps_per_s"] / out["fp64_plain"]["node_steps_per_s"]
    # compute roofline of the FP32 split step, counting the model's own operations: per Heun substep two
    # right-hand sides and the Heun update (y + dt r, then y + dt/2 (r + r2): 5 per state)
    meta = json.load(open(os.path.join(ROOT, "opendihu_b200/csrc/generated/"
                                             "shorten_ocallaghan_davidson_soboleva_2007_a32_c65.json")))
    n_sub = 2 * int(round(0.5 * system.dt_splitting / system.dt_0d))
    flops_node_step = n_sub * (2 * meta["operations_per_rhs"]["flops"] + 5 * meta["n_states"])
    achieved = out["fp32_reaction"]["node_steps_per_s"] * flops_node_step / 1e12
    fp32_peak = 148 * 128 * 2 * peaks()[1] * 1e6 / 1e12
    out["fp32_roofline"] = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                            "frac": achieved / fp32_peak, "flops_per_node_step": flops_node_step,
                            "peak_source": "derived: 148 SMs x 128 FP32 lanes x 2 flop x sm_max_mhz"}
    # accuracy on a sample over a span with action potentials
    grid = WL.shorten_grid(end_time=accuracy_ms)
    fires0 = np.nonzero(np.asarray(grid.firing_events)[0, np.asarray(grid.motor_unit_no) % grid.firing_events.shape[1]])[0]
    sample = WL.subset(grid, fires0[:16])
    nodes = ACC.traced_nodes(sample, 32)
    res = {}
    for name, prec in (("fp64", "fp64"), ("fp32", "fp32")):
        with S.FastMonodomainSolver(sample.copy(), method="split", precision=prec, device=device, trace_nodes=nodes,
                                    trace_capacity=0) as sv:
            sv.record_activation(0.0, 16)
            sv.advanceTimeSpan()
            res[name] = (sv.states()[0], *sv.activation_steps())
    out["accuracy"] = {"sample": "%d fibers x 1481 nodes (motor units firing at t = 0), %g ms (%d Strang steps)" % (
                           sample.n_fibers, accuracy_ms, int(round(accuracy_ms / sample.dt_splitting))),
                       "vm_max_abs_diff_fp32_vs_fp64_mV": float(np.max(np.abs(res["fp32"][0] - res["fp64"][0]))),
                       "vm_range_fp64_mV": [float(res["fp64"][0].min()), float(res["fp64"][0].max())],
                       "activation": ACC.compare_activation(res["fp32"][1], res["fp32"][2], res["fp64"][1],
                                                            res["fp64"][2])}
    out["method"] = "split path (the 56 states stay in the reaction kernel's registers over each half step)"
    return out


def c5_measurement(device: int, span_ms: float = 0.5, adjoint_steps: int = 4, subset_fibers: int = 16) -> dict:
    """Shorten 2007 at scale with the three extensions, over a bounded span: 10,000 fibers of U[1000,2500]
    nodes (17.5M nodes), 200 motor units, FP32 reaction with the autotuned method and launch shape, span_ms of
    simulated time (the configuration's 100 ms take hours at this size); Vm after the span against the FP64
    split solver on subset_fibers fibers of the system (same clamp nodes); and the FP64 adjoint of the sigma
    field (loss 1/2 sum of Vm^2 at 32 sensors per fiber over the last adjoint_steps Strang steps) with the
    memory plan of plan_adjoint for this device: checkpoint interval and sequential fiber shards."""
    import torch
    from opendihu_b200 import sharding as SH
    from opendihu_b200 import solver as S
    from opendihu_b200 import workloads as WL
    from opendihu_b200 import accuracy as ACC
    system = WL.shorten_scale(end_time=span_ms)
    dt = system.dt_splitting
    t_adj = span_ms - adjoint_steps * dt
    out = {"workload": "Shorten 2007, %d fibers x U[1000,2500] (%d nodes), 200 MUs, dt0D 1e-5, dt_split 5e-4, "
                       "%g ms" % (system.n_fibers, system.n_nodes, span_ms)}
    with S.FastMonodomainSolver(system.copy(), method="auto", precision="fp32", device=device) as sv:
        sv.setTimeSpan(0.0, 0.01)
        sv.advanceTimeSpan()
        sv.reset_timing()
        n0 = sv.split_steps()
        sv.setTimeSpan(0.01, t_adj)
        sv.advanceTimeSpan()
        states_adj = sv.states()
        sv.setTimeSpan(t_adj, span_ms)
        sv.advanceTimeSpan()
        ms = sv.timing()["advance_ms"]
        steps = sv.split_steps() - n0
        vm32 = sv.vm()
        out["fp32_forward"] = {"node_steps_per_s": system.n_nodes * steps / (ms / 1e3), "ms": ms,
                               "strang_steps": steps, "method": sv.method,
                               "tuning": {k: (sv.tuning or {}).get(k) for k in ("method", "steps_per_launch")}}
    sub = np.unique(np.linspace(0, system.n_fibers - 1, subset_fibers).round().astype(np.int64))
    ssys = WL.subset(system, sub)
    with S.FastMonodomainSolver(ssys, method="split", precision="fp64", device=device) as sv:
        sv.clamp_override = SH.shard_clamp_nodes(system, sub, SH.global_clamp_nodes(system))
        sv.advanceTimeSpan()
        vm64 = sv.vm()
    vm32_sub = vm32[SH.node_index(system.fiber_offsets, sub)]
    out["accuracy"] = {"sample": "%d fibers (%d nodes), FP64 split, same clamp nodes" % (len(sub), ssys.n_nodes),
                       "vm_max_abs_diff_fp32_vs_fp64_mV": float(np.max(np.abs(vm32_sub - vm64))),
                       "vm_range_mV": [float(vm64.min()), float(vm64.max())]}
    del vm32, vm32_sub
    # adjoint of sigma over the last Strang steps, from the FP32 run's state
    win = system.copy()
    win.states = states_adj
    win.start_time, win.end_time = t_adj, span_ms
    free, _ = torch.cuda.mem_get_info(device)
    budget = 0.6 * free
    plan = SH.plan_adjoint(win, t_adj, span_ms, budget)
    sensors = ACC.traced_nodes(win, 32)
    with S.FastMonodomainSolver(win, method="split", precision="fp64", device=device) as fw:
        fw.advanceTimeSpan()        # warm-up (module load, factorization)
        fw.reset_timing()
        fw.rewind()
        fw.set_states(states_adj)
        fw.advanceTimeSpan()
        fwd_ms = fw.timing()["advance_ms"]
    sh = SH.ShardedSolver(win, devices=(device,), n_shards=plan["n_shards"], method="split", precision="fp64")
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    trace, grads = sh.adjoint(t_adj, span_ms, plan["checkpoint_every"], sensors, lambda tr, cols: tr)
    torch.cuda.synchronize(device)
    adj_s = time.perf_counter() - t0
    dev = dict(sh.adjoint_device_ms)
    adj_dev_ms = dev["checkpointed_forward_ms"] + dev["backward_ms"]
    sh.close()
    out["adjoint"] = {"window": "%d Strang steps [%g, %g] ms, %d sensors, loss 1/2 sum Vm^2" % (
                          plan["n_steps"], t_adj, span_ms, len(sensors)),
                      "plan": {k: plan[k] for k in ("checkpoint_every", "n_shards", "bytes_per_node",
                                                    "largest_shard_nodes")},
                      "budget_bytes": budget, "peak_bytes_estimate": plan["largest_shard_nodes"] * plan["bytes_per_node"],
                      "fp64_forward_ms": fwd_ms, **dev,
                      "adjoint_over_forward": adj_dev_ms / fwd_ms,
                      "adjoint_wall_ms": adj_s * 1e3, "adjoint_wall_over_forward": adj_s * 1e3 / fwd_ms,
                      "timing": "CUDA events: one FP64 advance of the window (forward) against the checkpointed "
                                "forwards plus backward sweeps of all shards (adjoint); adjoint_wall_ms adds the "
                                "host work between shards (set-up, state upload, gradient download)",
                      "grad_sigma_norm": float(np.linalg.norm(grads["prefactor"] / (WL.AM * 0.58)))}
    return out


def emg_measurement(device: int, peak_hbm: float, cg_mesh=(97, 97, 297), cg_iterations: int = 160,
                    coupled: bool = True):
    """Coupled fibers + EMG (13 x 13 HH fibers x 1481 nodes, 25 x 25 x 149 3D nodes, one bidomain solve per
    1 ms coupling step, FP32 fused fibers) and the CG iteration on a 97 x 97 x 297 mesh (2.8M nodes)."""
    out = {}
    solver_cfg = {"relativeTolerance": 1e-8, "absoluteTolerance": 1e-30, "maxIterations": 20000}
    if coupled:
        out["coupled"] = emg_coupled(device, solver_cfg)
        seq = emg_coupled(device, solver_cfg, overlap=False)
        out["coupled"]["sequential_ms_per_coupling_step"] = seq["ms_per_coupling_step"]
    _cg_iteration(out, device, peak_hbm, cg_mesh, cg_iterations, solver_cfg)
    return out


def emg_coupled(device: int, solver_cfg: dict, overlap: bool = True) -> dict:
    import torch
    from opendihu_b200 import emg as E
    from opendihu_b200 import solver as S
    from opendihu_b200 import workloads as WL
    system, fpos, kw = WL.emg_box(n_fibers_x=13, n_fibers_y=13, n_nodes=1481, mesh_nodes=(25, 25, 149), end_time=5.0)
    fib = S.FastMonodomainSolver(system, method="fused", precision="fp32", device=device, autotune=True)
    bid = E.StaticBidomainSolver(emg_solver=solver_cfg, potential_flow_solver=solver_cfg, device=device, **kw)
    solves = []
    cp = E.Coupling(fib, bid, 1.0, 5.0, fpos, callback=lambda k, t, b: solves.append(b.timing()), overlap=overlap)
    with cp:
        cp.term1.setTimeSpan(0.0, 1.0)       # warm-up: one coupling step outside the timed span
        cp.term1.advanceTimeSpan()
        cp.term2.map_fibers(cp.term1)
        cp.term2.advanceTimeSpan()
        cp.start_time = 1.0
        solves.clear()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        cp.advanceTimeSpan()
        torch.cuda.synchronize(device)
        wall = time.perf_counter() - t0
        phi = cp.term2.phi_e()
        layout = fib.fused_layout()
        cpu = emg_cpu_baseline(cp.term2) if overlap else None
    return {
        "cpu_baseline": cpu,
        "workload": "fibers_emg-shaped box: 13 x 13 HH fibers x 1481 nodes (FP32 fused), 3D mesh 25 x 25 x 149 "
                    "nodes, sigma_i/sigma_e of the example, coupling dt 1 ms, CG rtol 1e-8",
        "coupling_steps": len(solves), "ms_per_coupling_step": wall / max(len(solves), 1) * 1e3,
        "emg_solve_ms": float(np.mean([t["solve_ms"] for t in solves])) if solves else None,
        "cg_iterations": [t["iterations"] for t in solves], "phi_e_max_abs": float(np.abs(phi).max()),
        "fiber_layout": layout,
        "overlap": overlap,
        "timing": "host wall clock around the coupled steps (fiber advance + transfer + solve; with overlap the "
                  "solve of step k runs beside the fiber advance of step k + 1)"}


def emg_cpu_baseline(bid) -> dict:
    """The last bidomain system solved on the host cores: scipy's conjugate gradients with the Jacobi
    preconditioner on the same matrix (the device-assembled stencil as CSR) and right-hand side, from zero,
    against the device solve from zero."""
    import scipy.sparse.linalg as spla
    sys.path.insert(0, ROOT)
    from oracle import emg_oracle as EO
    A = EO.stencil_to_sparse(bid.stencil(1), bid.shape).tocsr()
    b = bid.rhs()
    b = b - b.mean()
    dinv = 1.0 / A.diagonal()
    M = spla.LinearOperator(A.shape, matvec=lambda v: dinv * v)
    its = [0]

    def count(_):
        its[0] += 1
    t0 = time.perf_counter()
    x, info = spla.cg(A, b, rtol=1e-8, atol=0.0, maxiter=20000, M=M, callback=count)
    cpu_s = time.perf_counter() - t0
    x -= x.mean()
    keep = bid.initial_guess_nonzero
    bid.initial_guess_nonzero = False
    bid.advanceTimeSpan()
    bid.initial_guess_nonzero = keep
    t = bid.timing()
    phi = bid.phi_e()
    return {"kind": "port", "cores": 1, "solver": "scipy.sparse.linalg.cg, Jacobi preconditioner, rtol 1e-8, from 0",
            "cpu_solve_ms": cpu_s * 1e3, "cpu_iterations": its[0], "gpu_solve_ms_from_zero": t["solve_ms"],
            "gpu_iterations_from_zero": t["iterations"], "speedup": cpu_s * 1e3 / t["solve_ms"],
            "max_abs_diff": float(np.max(np.abs(phi - x)))}


def _cg_iteration(out: dict, device: int, peak_hbm: float, cg_mesh, cg_iterations: int, solver_cfg: dict):
    """CG iteration of the bidomain solve against the HBM roofline (mesh larger than L2)."""
    from opendihu_b200 import emg as E
    from opendihu_b200 import workloads as WL
    _, _, kw2 = WL.emg_box(n_fibers_x=2, n_fibers_y=2, n_nodes=1481, mesh_nodes=tuple(cg_mesh), width=3.0)
    z = kw2["node_positions"][:, 2]
    vm = -75.0 + 100.0 * np.exp(-((z - z.mean()) / 0.3) ** 2)
    with E.StaticBidomainSolver(emg_solver={"relativeTolerance": 1e-30, "absoluteTolerance": 0.0,
                                            "maxIterations": cg_iterations},
                                potential_flow_solver=solver_cfg, device=device, preconditioner="jacobi",
                                **kw2) as big:
        big.set_vm(vm)
        big.advanceTimeSpan()
        big.initial_guess_nonzero = False
        big.advanceTimeSpan()
        t = big.timing()
        n = big.n_nodes
    # the whole solve to rtol 1e-8 from a zero initial guess with either preconditioner
    solves = {}
    for pc in ("jacobi", "multigrid"):
        with E.StaticBidomainSolver(emg_solver=solver_cfg, potential_flow_solver=solver_cfg, device=device,
                                    preconditioner=pc, initial_guess_nonzero=False, **kw2) as sv:
            sv.set_vm(vm)
            sv.advanceTimeSpan()
            sv.advanceTimeSpan()
            tt = sv.timing()
            solves[pc] = {"solve_ms": tt["solve_ms"], "iterations": tt["iterations"], "levels": sv.multigrid_levels}
    per_it_ms = t["solve_ms"] / max(t["iterations"], 1)
    # algorithmic bytes per node and iteration: direction pass (14 stencil coefficients, z, p and q read, p and
    # q written: 152 B) + update pass (x, r read and written, p, q, dinv read, z written: 64 B)
    bytes_it = 216 * n
    gbs = bytes_it / (per_it_ms / 1e3) / 1e9
    out["cg_iteration"] = {"workload": "%d x %d x %d mesh (%d nodes), %d iterations" % (*cg_mesh, n, cg_iterations),
                           "iterations": t["iterations"], "preconditioner": "jacobi",
                           "solve_to_rtol_1e-8": solves,
                           "solve_ms": t["solve_ms"], "ms_per_iteration": per_it_ms,
                           "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak_hbm, "unit": "GB/s",
                                        "frac": gbs / peak_hbm, "algorithmic_bytes_per_node_iteration": 216,
                                        "timing": "CUDA events around the solve (includes the host checks every "
                                                  "8 iterations)"}}


def workload_config(args, world: int) -> dict:
    """The benchmark workload, the same dict in both arms (the implementation is described beside it)."""
    return {"workload": "batched_hh: %d HH fibers/GPU, lengths U[500,2500] (seed=rank), 100 MUs, Poisson 10-40 Hz, "
                        "Crank-Nicolson, dt0D 1e-4 ms, dt_split 1e-3 ms" % args.fibers,
            "step": "%g ms = %d Strang steps" % (args.step_ms, int(round(args.step_ms / 1e-3))),
            "l2": "inputs larger than L2", "parallelism": "fibers sharded, %d GPU(s), no collective" % world}


def run_reference(args):
    world, rank, local, pg = dist_setup(args)
    if rank != 0:
        return
    from opendihu_b200 import workloads as WL
    system = WL.batched_hh(n_fibers=args.fibers, seed=0)
    threads = os.cpu_count() or 1
    times = []
    for k in range(args.warmup + args.steps):
        _, _, n, rate, dt = cpu_baseline(system, threads, 0.2, threads)   # one fiber per host thread
        if k >= args.warmup:
            times.append(rate)
    value = float(np.median(times))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "node-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload_config(args, world),
            "implementation": "CPU oracle port of the reference's vc FastMonodomainSolver (the reference needs "
                              "PETSc/MPI/Vc and cannot be built here), one fiber per host thread",
            "cpu_baseline": {"value": value, "unit": "node-steps/s", "cores": threads, "kind": "port",
                             "sample": f"each step the first {threads} fibers of the batch over 0.2 ms"},
            "e2e": {"value": value, "unit": "node-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def side_line(name: str, value) -> None:
    """A side measurement as its own JSON line (printed before the headline line)."""
    print(json.dumps({"side": name, name: value}), flush=True)


def side(name: str, fn):
    """Runs one side measurement and prints its line; a failure is printed as the measurement's error and does
    not stop the benchmark (the headline line is printed regardless)."""
    try:
        value = fn()
    except Exception as e:  # noqa: BLE001 - reported, the headline still follows
        import traceback
        print(json.dumps({"side": name, "error": f"{type(e).__name__}: {e}",
                          "where": traceback.format_exc().strip().splitlines()[-3:]}), flush=True)
        return None
    side_line(name, value)
    return value


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    world, rank, local, pg = dist_setup(args)
    from opendihu_b200 import accuracy as ACC
    from opendihu_b200 import solver as S
    from opendihu_b200 import workloads as WL
    if world > 1:
        # the side measurements (plain configuration, adjoint, EMG, Shorten, accuracy and CPU baseline) are
        # single-GPU numbers reported by the 1-GPU run; on N GPUs rank 0 would hold the other GPUs meanwhile
        args.skip_adjoint = args.skip_emg = args.skip_shorten = args.skip_accuracy = args.skip_c5 = True
    cg_mesh = tuple(int(x) for x in args.emg_cg_mesh.split(","))
    if args.only:
        if rank == 0:
            if args.only in ("emg", "emg-cg"):
                out = {"emg": emg_measurement(local, peaks()[0], cg_mesh, args.emg_cg_iterations,
                                              coupled=args.only == "emg")}
            elif args.only == "plain":
                out = {"plain_config_node_steps_per_s": plain_measurement(
                    local, args.plain_legs.split(",") if args.plain_legs else None)}
            elif args.only == "adjoint":
                out = {"adjoint": adjoint_measurement(local, args.adjoint_ms)}
            elif args.only == "c5":
                out = {"c5": c5_measurement(local, args.c5_ms, args.c5_adjoint_steps)}
            elif args.only == "c2-accuracy":
                out = {"c2_accuracy": ACC.batch_accuracy(WL.batched_hh(n_fibers=args.fibers, seed=0), local,
                                                         args.accuracy_ms)}
            else:
                out = {"shorten": shorten_measurement(local, args.shorten_ms, args.shorten_accuracy_ms)}
            print(json.dumps(out), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return

    system = WL.batched_hh(n_fibers=args.fibers, seed=rank)
    n_nodes = system.n_nodes
    fused = S.FastMonodomainSolver(system.copy(), method="fused", precision="fp32", profile=True, device=local,
                                   threads_per_block=args.threads, nodes_per_thread=args.nodes_per_thread,
                                   steps_per_launch=args.steps_per_launch, autotune=not args.no_autotune)
    fused.initialize()
    tuning = fused.tuning
    step = args.step_ms
    t = 0.0
    for _ in range(args.warmup):
        fused.setTimeSpan(t, t + step)
        fused.advanceTimeSpan()
        t += step
    barrier(pg)
    fused.reset_timing()
    n0 = fused.split_steps()
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.steps):
        fused.setTimeSpan(t, t + step)
        fused.advanceTimeSpan()
        t += step
    clk = clocks.stop()
    tm = fused.timing()
    split_steps = fused.split_steps() - n0
    dev_s = tm["advance_ms"] / 1e3
    dev_s_max = allmax(pg, dev_s)
    node_steps_rank = n_nodes * split_steps
    value = node_steps_rank * world / dev_s_max
    kernel_avg_ms = tm["main_kernel_ms"] / max(tm["main_kernel_launches"], 1)
    launches_per_kernel = tm["main_kernel_launches"]
    steps_per_launch = split_steps / max(launches_per_kernel, 1)

    # end to end through the public API with host buffers, over the same K steps: H2D of the states from
    # page-locked host memory, the advance, D2H of the states, every step
    host_states = fused.states(out=fused.pinned_states())
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fused.set_states(host_states)
        fused.setTimeSpan(t, t + step)
        fused.advanceTimeSpan()
        host_states = fused.states(out=host_states)
        t += step
    e2e_s = allmax(pg, time.perf_counter() - t0)
    e2e_value = n_nodes * split_steps * world / e2e_s
    state_bytes = n_nodes * 8 * 4
    fused_shape = {"threads": fused.threads_per_block, "nodes_per_thread": fused.nodes_per_thread,
                   "cluster_size": fused.cluster_size, "steps_per_launch": steps_per_launch,
                   "autotuned": tuning is not None}
    fused.close()

    # FP64 split ("plain") and FP64 fused solvers on the same batch: the first is the reference's method, the
    # second separates the gain of fusion from the gain of the FP32 reaction
    fp64 = {}
    if not args.skip_fp64:
        for name, method in (("split", "split"), ("fused", "fused")):
            slv = S.FastMonodomainSolver(system.copy(), method=method, precision="fp64", device=local,
                                         autotune=method == "fused")
            slv.initialize()
            tp = 0.0
            slv.setTimeSpan(tp, tp + step)
            slv.advanceTimeSpan()
            tp += step
            barrier(pg)
            slv.reset_timing()
            p0 = slv.split_steps()
            for _ in range(2):
                slv.setTimeSpan(tp, tp + step)
                slv.advanceTimeSpan()
                tp += step
            p_s = allmax(pg, slv.timing()["advance_ms"] / 1e3)
            fp64[name] = n_nodes * (slv.split_steps() - p0) * world / p_s
            slv.close()

    # side measurements, each printed as its own line before the headline line
    plain_cfg = adj = acc = cpu = None
    if rank == 0 and not args.skip_fp64 and world == 1:
        plain_cfg = side("plain_config_node_steps_per_s", lambda: plain_measurement(local))
    if rank == 0 and not args.skip_adjoint:
        adj = side("adjoint", lambda: adjoint_measurement(local, args.adjoint_ms))
    if rank == 0 and not args.skip_emg:
        side("emg", lambda: emg_measurement(local, peaks()[0], cg_mesh, args.emg_cg_iterations))
    if rank == 0 and not args.skip_shorten:
        side("shorten", lambda: shorten_measurement(local, args.shorten_ms, args.shorten_accuracy_ms))
    if rank == 0 and not args.skip_c5:
        side("c5", lambda: c5_measurement(local, args.c5_ms, args.c5_adjoint_steps))
    if rank == 0 and not args.skip_accuracy:
        acc = side("c2_accuracy", lambda: ACC.batch_accuracy(system, local, args.accuracy_ms, chunk_ms=2.0))
        # the oracle's CPU throughput on a bounded sample of the batch, all host threads, and one thread (the
        # reference's vc path runs one thread per MPI rank)
        threads = os.cpu_count() or 1
        # one fiber per host thread (the oracle parallelizes over fibers)
        sub, ref, n_ref, rate, cpu_s = cpu_baseline(system, threads, 10.0, threads)
        cpu = {"value": rate, "unit": "node-steps/s", "cores": threads, "kind": "port",
               "sample": f"first {threads} fibers of the batch ({sub.n_nodes} nodes) x 10 ms ({n_ref} Strang "
                         f"steps), one fiber per thread, {cpu_s:.1f} s"}
        sub1, _, n1, rate1, cpu1_s = cpu_baseline(system, 1, 10.0, 1)
        cpu["single_thread"] = {"value": rate1, "cores": 1,
                                "sample": f"first fiber ({sub1.n_nodes} nodes) x 10 ms ({n1} Strang steps)"}

    peak_hbm, sm_max, peak_kind = peaks()
    ops = hh_ops()
    n0d = 5
    fp32_flops_node_step = 2 * n0d * (2 * ops["flops"] + 6 + 9)
    # algorithmic HBM bytes of one fused launch, per node: states read and written once (Vm f64, 3 gates and
    # their 3 compensation residuals f32), 3 parameters (f32), 6 diffusion coefficients (f64), clamp map (i32)
    bytes_launch = n_nodes * (2 * (8 + 12 + 12) + 12 + 48 + 4)
    achieved_gbs = bytes_launch / (kernel_avg_ms / 1e3) / 1e9 if kernel_avg_ms > 0 else None
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12
    achieved_tf = (n_nodes * steps_per_launch * fp32_flops_node_step / (kernel_avg_ms / 1e3) / 1e12
                   if kernel_avg_ms > 0 else None)
    traffic = None
    prof = os.path.join(ROOT, "profiles", "fused_kernel_batched_hh.md")
    if os.path.exists(prof):
        for ln in open(prof):
            if ln.startswith("dram_bytes_per_node_per_launch:"):
                traffic = float(ln.split(":", 1)[1]) * n_nodes

    if rank == 0:
        acc_line = None
        if acc:
            a32 = acc["fp32_fused_vs_fp64_fused"]
            acc_line = {"span_ms": args.accuracy_ms, "fibers": system.n_fibers,
                        "vm_max_abs_mV": a32["vm_max_abs_diff_mV"],
                        "activation_max_step_diff": a32["activation"]["max_step_diff"],
                        "activation_nodes_count_mismatch": a32["activation"]["nodes_count_mismatch"],
                        "crossings": a32["activation"]["crossings"],
                        "traced_nodes": a32["activation"]["traced_nodes"],
                        "fp64_split_vs_fused_vm_max_abs_mV": acc["fp64_split_vs_fp64_fused"]["vm_max_abs_diff_mV"],
                        "reference": "FP64 fused, all fibers; FP64 split on %d fibers" % (
                            acc["fp64_split_vs_fp64_fused"]["fibers"])}
        line = {
            "metric": METRIC, "value": value, "unit": "node-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_s_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 reaction + f64 Vm/diffusion",
            "data": "synthetic (seeded)",
            "config": workload_config(args, world),
            "implementation": {"method": "fused persistent kernel, FP32 reaction", "n_nodes_per_gpu": n_nodes,
                               "fused_shape": fused_shape},
            "e2e": {"value": e2e_value, "unit": "node-steps/s", "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "steps": args.steps},
            "gpu_launches": int(tm["kernel_launches"]),
            "roofline_hbm": {"achieved": achieved_gbs, "peak": peak_hbm, "unit": "GB/s",
                             "frac": (achieved_gbs / peak_hbm) if achieved_gbs else None, "peak_source": peak_kind},
            "cpu_baseline": cpu,
            "clocks": clk,
            # the north-star ratios last, so that the end of the line (what a log tail keeps) holds them
            "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": (achieved_tf / fp32_peak) if achieved_tf else None, "traffic": traffic,
                         "peak_source": "derived (148 SMs x 128 lanes x 2 x sm_max_mhz)",
                         "kernel": "fused_kernel %.3f ms/launch, %.0f steps/launch" % (kernel_avg_ms, steps_per_launch)},
            "fp64_fused": {"value": fp64.get("fused"), "speedup": (value / fp64["fused"]) if fp64.get("fused") else None},
            "accuracy_vs_fp64": acc_line,
            "adjoint_over_forward": adj["adjoint_over_forward"] if adj else None,
            "fp64_plain": {"value": fp64.get("split"), "speedup": (value / fp64["split"]) if fp64.get("split") else None},
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
