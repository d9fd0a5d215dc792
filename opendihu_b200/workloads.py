"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference's large example inputs (fiber geometry files, MU_firing_times_real.txt,
MU_fibre_distribution_3780.txt) are not available; these generators stand in for them with the
stated shapes and distributions, written in the reference's file formats where files are needed.
All fibers are straight with uniform element length dx.
"""
from __future__ import annotations

import numpy as np

from . import inputs
from .sharding import subset  # noqa: F401  (re-exported: the given fibers as a system)
from .solver import FiberSystem, uniform_fibers

HH = "hodgkin_huxley_1952"
SHORTEN = "shorten_ocallaghan_davidson_soboleva_2007"

SIGMA = 3.828   # mS/cm
AM = 500.0      # 1/cm
CM = 1.0        # uF/cm^2


def plain_hh(n_fibers: int = 16, n_nodes: int = 1481, end_time: float = 10.0, **kw) -> FiberSystem:
    """Plain-method configuration: HH, identical fibers of 1481 nodes (14.8 cm), dx 0.01 cm,
    prefactor sigma/(Am*Cm), Heun dt 1e-4 ms, implicit Euler / Strang dt 1e-3 ms, clamp stimulus at the
    centre for 0.1 ms every 10 ms."""
    return uniform_fibers(HH, [n_nodes] * n_fibers, 0.01, SIGMA / (AM * CM), call_frequency=0.1,
                          repeat_after_first_call=0.1, call_enable_begin=0.0, end_time=end_time, dt_0d=1e-4,
                          dt_1d=1e-3, dt_splitting=1e-3, dt_repeated_call=1e-3, **kw)


def batched_hh(n_fibers: int = 4096, min_nodes: int = 500, max_nodes: int = 2500, n_mus: int = 100,
               end_time: float = 100.0, seed: int = 0, **kw) -> FiberSystem:
    """Batching + precision configuration: HH, fiber lengths uniform in [500, 2500] nodes (seeded),
    dx 0.01 cm, fibers assigned to 100 motor units by a seeded exponential size distribution, per-MU
    Poisson firing at 10-40 Hz sampled at the 0.1/ms call frequency, Crank-Nicolson, dt as the plain
    configuration, junction = NMJ node and its two neighbours of each fiber."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(min_nodes, max_nodes + 1, size=n_fibers)
    mus = inputs.exponential_mu_distribution(n_fibers, n_mus, seed)
    firing = inputs.poisson_firing_times(n_mus, end_time, 0.1, 10.0, 40.0, seed)
    kw.setdefault("diffusion_scheme", "CrankNicolson")
    # fibers of uneven length: each fiber's junction is its own NMJ node and its two neighbours (the rule of the
    # reference's GPU path); the vc path's rule attributes point buffers to fibers as if all had the length of
    # the first (fast_monodomain_solver_compute.tpp:158-161) and would leave most junctions unstimulated
    kw.setdefault("clamp_rule", "center")
    return uniform_fibers(HH, lengths, 0.01, SIGMA / (AM * CM), firing_events=firing, motor_unit_no=mus,
                          call_frequency=0.1, repeat_after_first_call=0.1, call_enable_begin=0.0,
                          end_time=end_time, dt_0d=1e-4, dt_1d=1e-3, dt_splitting=1e-3, dt_repeated_call=1e-3, **kw)


def shorten_grid(n_fibers: int = 1369, n_nodes: int = 1481, end_time: float = 50.0, n_mus: int = 100,
                 seed: int = 0, **kw) -> FiberSystem:
    """Shorten 2007 (56 states): 37x37 fibers x 1481 nodes, Heun dt 1e-5 ms, Strang dt 5e-4 ms,
    seeded per-MU firing."""
    mus = inputs.exponential_mu_distribution(n_fibers, n_mus, seed)
    firing = inputs.poisson_firing_times(n_mus, end_time, 0.1, 10.0, 40.0, seed)
    return uniform_fibers(SHORTEN, [n_nodes] * n_fibers, 0.01, SIGMA / (AM * 0.58), firing_events=firing,
                          motor_unit_no=mus, call_frequency=0.1, repeat_after_first_call=0.1, call_enable_begin=0.0,
                          end_time=end_time, dt_0d=1e-5, dt_1d=5e-4, dt_splitting=5e-4, dt_repeated_call=5e-4, **kw)


def shorten_scale(n_fibers: int = 10000, min_nodes: int = 1000, max_nodes: int = 2500, n_mus: int = 200,
                  end_time: float = 100.0, seed: int = 0, **kw) -> FiberSystem:
    """Shorten 2007 at scale: fiber lengths uniform in [1000, 2500] nodes (seeded), 200 motor units with
    exponential sizes, Poisson firing 10-40 Hz sampled at 0.1/ms, Heun dt 1e-5 ms, Strang dt 5e-4 ms."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(min_nodes, max_nodes + 1, size=n_fibers)
    mus = inputs.exponential_mu_distribution(n_fibers, n_mus, seed)
    firing = inputs.poisson_firing_times(n_mus, max(end_time, 0.1), 0.1, 10.0, 40.0, seed)
    kw.setdefault("clamp_rule", "center")   # uneven lengths: each fiber's own junction (see batched_hh)
    return uniform_fibers(SHORTEN, lengths, 0.01, SIGMA / (AM * 0.58), firing_events=firing, motor_unit_no=mus,
                          call_frequency=0.1, repeat_after_first_call=0.1, call_enable_begin=0.0,
                          end_time=end_time, dt_0d=1e-5, dt_1d=5e-4, dt_splitting=5e-4, dt_repeated_call=5e-4, **kw)


def differentiation_hh(n_fibers: int = 256, n_nodes: int = 1481, end_time: float = 20.0, n_sensors: int = 32,
                       seed: int = 1, **kw):
    """Differentiation configuration: HH, 256 fibers x 1481 nodes, per-fiber sigma ~ U[2.5, 5.0] mS/cm and
    per-fiber g_Na, g_K scaled by U[0.8, 1.2] (seeded), 32 sensor nodes per fiber evenly spaced, 20 ms.
    Returns (system, sigma, scale_na, scale_k, sensor_nodes); parameters slot 1 = g_Na, slot 2 = g_K."""
    rng = np.random.default_rng(seed)
    sigma = rng.uniform(2.5, 5.0, size=n_fibers)
    s_na = rng.uniform(0.8, 1.2, size=n_fibers)
    s_k = rng.uniform(0.8, 1.2, size=n_fibers)
    sysm = plain_hh(n_fibers=n_fibers, n_nodes=n_nodes, end_time=end_time, **kw)
    sysm.prefactor = sigma / (AM * CM)
    sysm.parameters = hh_parameters(sysm, s_na, s_k)
    idx = np.linspace(0, n_nodes - 1, n_sensors).round().astype(np.int64)
    sensors = (np.asarray(sysm.fiber_offsets[:-1])[:, None] + idx[None, :]).reshape(-1)
    return sysm, sigma, s_na, s_k, sensors


def hh_parameters(system: FiberSystem, s_na, s_k, i_stim: float = 0.0) -> np.ndarray:
    """Per-node HH parameter slots (I_Stim, g_Na, g_K) with per-fiber scales of the model's 120 and 36 mS/cm^2."""
    lengths = np.diff(np.asarray(system.fiber_offsets))
    p = np.zeros((3, system.n_nodes))
    p[0] = i_stim
    p[1] = np.repeat(120.0 * np.asarray(s_na), lengths)
    p[2] = np.repeat(36.0 * np.asarray(s_k), lengths)
    return p


# fibers_emg conductivities (settings_fibers_emg.py "Activation"): sigma_i in fiber coordinates, sigma_e
EMG_SIGMA_I = (8.93, 0.0, 0.0, 0.0, 0.893, 0.0, 0.0, 0.0, 0.893)
EMG_SIGMA_E = (6.7, 0.0, 0.0, 0.0, 6.7, 0.0, 0.0, 0.0, 6.7)


def emg_box(n_fibers_x: int = 13, n_fibers_y: int = 13, n_nodes: int = 1481, mesh_nodes=(25, 25, 149),
            width: float = 3.0, end_time: float = 10.0, n_mus: int = 10, seed: int = 0, **kw):
    """Fibers + EMG configuration in the shape of the fibers_emg example: a muscle box of width x width x
    (n_nodes - 1) * 0.01 cm with a grid of n_fibers_x x n_fibers_y HH fibers along z (dx 0.01 cm, seeded
    MU assignment and Poisson firing as batched_hh), a structured 3D mesh of mesh_nodes nodes over the box,
    potential-flow Dirichlet values 0 on the bottom face and 1 on the top face, the example's sigma_i and
    sigma_e.  Returns (system, fiber node positions [n, 3], StaticBidomainSolver keyword arguments)."""
    nf = n_fibers_x * n_fibers_y
    length = (n_nodes - 1) * 0.01
    mus = inputs.exponential_mu_distribution(nf, n_mus, seed)
    firing = inputs.poisson_firing_times(n_mus, end_time, 0.1, 10.0, 40.0, seed)
    system = uniform_fibers(HH, [n_nodes] * nf, 0.01, SIGMA / (AM * CM), firing_events=firing, motor_unit_no=mus,
                            call_frequency=0.1, repeat_after_first_call=0.1, call_enable_begin=0.0,
                            end_time=end_time, dt_0d=1e-4, dt_1d=1e-3, dt_splitting=1e-3, dt_repeated_call=1e-3, **kw)
    fx = (np.arange(n_fibers_x) + 0.5) * width / n_fibers_x
    fy = (np.arange(n_fibers_y) + 0.5) * width / n_fibers_y
    z = np.arange(n_nodes) * 0.01
    pos = np.concatenate([np.stack([np.full(n_nodes, x), np.full(n_nodes, y), z], axis=1)
                          for y in fy for x in fx])
    nx, ny, nz = mesh_nodes
    xs, ys, zs = np.linspace(0, width, nx), np.linspace(0, width, ny), np.linspace(0, length, nz)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    mesh = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    bottom = np.arange(nx * ny)
    top = np.arange(nx * ny) + nx * ny * (nz - 1)
    emg = dict(shape=(nx, ny, nz), node_positions=mesh, sigma_i=EMG_SIGMA_I, sigma_e=EMG_SIGMA_E,
               dirichlet_nodes=np.concatenate([bottom, top]),
               dirichlet_values=np.concatenate([np.zeros(nx * ny), np.ones(nx * ny)]))
    return system, pos, emg
