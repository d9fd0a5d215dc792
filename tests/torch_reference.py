"""FP64 reference gradient for the adjoint tests: the discrete forward (RepeatedCall / Strang / Heun with the
junction clamps / consistent-mass diffusion solve), written with PyTorch operations and differentiated by
autograd.  It is an independent implementation of the same discrete map the CUDA adjoint differentiates:
its forward is checked against the oracle, its gradients against the CUDA adjoint.  Small problems only
(dense per-fiber solves, one autograd graph node per operation)."""
from __future__ import annotations

import json
import math
import os

import numpy as np
import torch

import helpers as H
from opendihu_b200 import cellml

GEN = os.path.join(H.ROOT, "opendihu_b200", "csrc", "generated")


class TorchModel:
    def __init__(self, model: str):
        name = {H.HH: "hodgkin_huxley_1952_anone_c2_3_4", H.SHORTEN:
                "shorten_ocallaghan_davidson_soboleva_2007_a32_c65"}[model]
        meta = json.load(open(os.path.join(GEN, name + ".json")))
        self.n_states = meta["n_states"]
        self.consts = meta["constants"]
        self.lines = [(k, i, cellml.tree_from_json(t)) for k, i, t in meta["rhs_lines"]]

    def _powi(self, x, n):
        if n < 0:
            return 1.0 / self._powi(x, -n)
        if n == 1:
            return x
        if n == 2:
            return x * x
        e0 = n // 2
        e1 = n - e0
        if e0 == 1:
            return x * self._powi(x, e1)
        return self._powi(x, e0) * self._powi(x, e1)

    def _ev(self, e, env):
        t = e[0]
        if t == "num":
            return e[2]
        if t == "var":
            k, i = e[1], e[2]
            if k == "C":
                return self.consts[i]
            if k == "S":
                return env["S"][i]
            if k == "P":
                return env["P"][i]
            if k == "A":
                return env["A"][i]
            if k == "T":
                return env["T"]
            raise ValueError(k)
        if t == "neg":
            return -self._ev(e[1], env)
        if t == "pos":
            return self._ev(e[1], env)
        if t == "bin":
            a = self._ev(e[2], env)
            b = self._ev(e[3], env)
            op = e[1]
            if op == "+":
                return a + b
            if op == "-":
                return a - b
            if op == "*":
                return a * b
            if op == "/":
                return a / b
            cmp = {"<": torch.lt, "<=": torch.le, ">": torch.gt, ">=": torch.ge, "==": torch.eq, "!=": torch.ne}
            if op in cmp:
                return cmp[op](torch.as_tensor(a), torch.as_tensor(b))
            if op == "&&":
                return torch.logical_and(torch.as_tensor(a), torch.as_tensor(b))
            if op == "||":
                return torch.logical_or(torch.as_tensor(a), torch.as_tensor(b))
        if t == "tern":
            c = self._ev(e[1], env)
            return torch.where(torch.as_tensor(c), torch.as_tensor(self._ev(e[2], env), dtype=torch.float64),
                               torch.as_tensor(self._ev(e[3], env), dtype=torch.float64))
        if t == "call":
            f = e[1]
            if f == "pow":
                n = cellml._int_exponent(e[2][1])
                x = self._ev(e[2][0], env)
                if n is not None:
                    return self._powi(x, n)
                return torch.pow(torch.as_tensor(x), self._ev(e[2][1], env))
            x = torch.as_tensor(self._ev(e[2][0], env), dtype=torch.float64)
            return {"exp": torch.exp, "log": torch.log, "fabs": torch.abs, "sqrt": torch.sqrt}[f](x)
        raise ValueError(e)

    def rates(self, t, y, P):
        env = {"S": y, "P": P, "A": {}, "T": t}
        r = [None] * self.n_states
        for k, i, e in self.lines:
            v = self._ev(e, env)
            if k == "A":
                env["A"][i] = v
            else:
                r[i] = v
        return r


class Tss:
    def __init__(self, start, end, dt):
        self.start, self.end, self.dt, self.target, self.n = start, end, dt, dt, 1

    def set_dt(self, dt):
        self.target = dt
        self.n = max(1, int(math.ceil((self.end - self.start) / dt - 0.1)))
        self.dt = (self.end - self.start) / self.n

    def set_span(self, s, e):
        self.start, self.end = s, e
        if self.target > e - s:
            self.dt = e - s
        self.set_dt(self.dt)


def plan(system):
    """(t, mid, dt0, n0, dt1) of every Strang step, by the reference's time rules."""
    rc = Tss(system.start_time, system.end_time, system.dt_repeated_call)
    rc.set_dt(system.dt_repeated_call)
    span = rc.end - rc.start
    st = Tss(system.start_time, system.start_time + system.dt_splitting, system.dt_splitting)
    he = Tss(system.start_time, system.start_time + system.dt_0d, system.dt_0d)
    di = Tss(system.start_time, system.start_time + system.dt_1d, system.dt_1d)
    out = []
    t = rc.start
    for k in range(rc.n):
        st.set_span(t, t + rc.dt)
        start, dts, ns = st.start, st.dt, st.n
        he.set_span(start, start + 0.5 * dts)
        di.set_span(start, start + dts)
        for j in range(ns):
            tc = start + j * dts
            out.append((tc, tc + 0.5 * dts, he.dt, he.n, di.dt))
        t = rc.start + (k + 1) / rc.n * span
    return out


class Machine:
    """The stimulation machine of one fiber (fast_monodomain_solver_compute.tpp:509-627)."""

    def __init__(self, system, f):
        self.freq = system.call_frequency[f]
        self.rep = system.repeat_after_first_call[f]
        self.beg = system.call_enable_begin[f]
        self.jit_vals = np.asarray(system.jitter)[f] if system.jitter is not None and np.asarray(system.jitter).size else []
        self.mu = int(system.motor_unit_no[f])
        self.fe = np.asarray(system.firing_events)
        self.jit = 0.0
        self.jidx = 0
        self.last = self.beg - 1e-13 - 1.0 / (self.freq + self.jit)

    def __call__(self, t):
        check = False
        if t >= self.last + 1.0 / (self.freq + self.jit) and t >= self.beg - 1e-13:
            check = True
            if self.rep != 0 and t - (self.last + 1.0 / (self.freq + self.jit)) > self.rep:
                self.last += 1.0 / (self.freq + self.jit)
                jf = self.jit_vals[self.jidx % len(self.jit_vals)] if len(self.jit_vals) else 0.0
                self.jit = jf * self.freq
                self.jidx += 1
                check = False
        idx = int(np.floor(abs(t * self.freq) + 0.5)) * (1 if t * self.freq >= 0 else -1)
        row = idx % self.fe.shape[0]
        return check and bool(self.fe[row, self.mu % self.fe.shape[1]])


def forward(system, prefactor, params, sensors, clamp_first, clamp_count, gate_codes=None):
    """Differentiable trace [steps, sensors]; prefactor [n_fibers] and params [n_params, n_nodes] are torch
    tensors (float64), states start from system.states.  gate_codes (per node attributed fiber * 4 + class,
    from the library's host-only selection): onlyComputeIfHasBeenStimulated, a node keeps its state at the
    substeps its attributed fiber's flag does not yet allow (compute.tpp:201-205 in buffer order)."""
    model = TorchModel(system.model)
    off = np.asarray(system.fiber_offsets)
    nf = len(off) - 1
    N = int(off[-1])
    y = [torch.as_tensor(system.states[s], dtype=torch.float64) for s in range(model.n_states)]
    P = [params[q] for q in range(params.shape[0])]
    machines = [Machine(system, f) for f in range(nf)]
    clamp_nodes = [list(range(clamp_first[f], clamp_first[f] + clamp_count[f])) if clamp_first[f] >= 0 else []
                   for f in range(nf)]
    vstim = system.value_for_stimulated_point
    ie = system.diffusion_scheme == "ImplicitEuler"
    h_all = np.asarray(system.element_lengths)
    trace = []
    sensors_t = torch.as_tensor(np.asarray(sensors), dtype=torch.long)

    evaluated = [len(c) > 0 for c in clamp_nodes]
    hbs = [False] * nf

    def half(t0, dt0, n0, y):
        stims = []
        for k in range(n0):
            t = t0 + k * dt0
            stims.append([machines[f](t) if evaluated[f] else False for f in range(nf)])
        first = np.zeros(N, np.int64)
        if gate_codes is not None:
            start = []
            for f in range(nf):
                ks = [k for k in range(n0) if stims[k][f]]
                start.append(0 if hbs[f] else (ks[0] + 1 if ks else 255))
                hbs[f] = hbs[f] or bool(ks)
            for i in range(N):
                st, cls = start[gate_codes[i] >> 2], gate_codes[i] & 3
                first[i] = st if st in (0, 255) else (st - 1 if cls == 1 else (255 if cls == 0 else 0))
        for k in range(n0):
            t = t0 + k * dt0
            mask = np.zeros(N, bool)
            for f in range(nf):
                if stims[k][f]:
                    mask[clamp_nodes[f]] = True
            m = torch.as_tensor(mask)
            r = model.rates(t, y, P)
            ys = [y[s] + dt0 * r[s] for s in range(model.n_states)]
            ys[0] = torch.where(m, torch.full_like(ys[0], vstim), ys[0])
            r2 = model.rates(t, ys, P)
            yn = [y[s] + 0.5 * dt0 * (r[s] + r2[s]) for s in range(model.n_states)]
            yn[0] = torch.where(m, torch.full_like(yn[0], vstim), yn[0])
            on = torch.as_tensor(k >= first)
            y = [torch.where(on, yn[s], y[s]) for s in range(model.n_states)]
        return y

    def diffusion(u, dt):
        parts = []
        for f in range(nf):
            n = off[f + 1] - off[f]
            h = torch.as_tensor(h_all[off[f] - f:off[f + 1] - f - 1], dtype=torch.float64)
            k = prefactor[f] / h
            mo = h / 6
            md = h / 3
            if ie:
                oa, da, ob, db = k - mo / dt, -k - md / dt, -mo / dt, -md / dt
            else:
                oa, da, ob, db = k / 2 - mo / dt, -k / 2 - md / dt, -k / 2 - mo / dt, k / 2 - md / dt
            z = torch.zeros(1, dtype=torch.float64)
            dA = torch.cat([da, z]) + torch.cat([z, da])
            dB = torch.cat([db, z]) + torch.cat([z, db])
            A = torch.diag(dA) + torch.diag(oa, 1) + torch.diag(oa, -1)
            B = torch.diag(dB) + torch.diag(ob, 1) + torch.diag(ob, -1)
            uf = u[off[f]:off[f + 1]]
            parts.append(torch.linalg.solve(A, B @ uf))
        return torch.cat(parts)

    for (t, mid, dt0, n0, dt1) in plan(system):
        y = half(t, dt0, n0, y)
        y[0] = diffusion(y[0], dt1)
        y = half(mid, dt0, n0, y)
        trace.append(y[0][sensors_t])
    return torch.stack(trace), y


