"""Fibers -> 3D static bidomain (EMG): the caller downstream of the fiber solver.

Mirrors the reference's operators of the fibers_emg example (examples/electrophysiology/fibers/fibers_emg/
src/fast_fibers_emg.cpp:17-63):

* ``StaticBidomainSolver`` -- TimeSteppingScheme::StaticBidomainSolver (core/src/specialized_solver/
  static_bidomain_solver.tpp): at initialisation the "PotentialFlow" Laplace problem gives the fiber
  direction; every ``advanceTimeSpan`` solves K(sigma_i + sigma_e) phi_e = -K(sigma_i) Vm on the 3D mesh.
* ``Coupling`` -- Control::Coupling (core/src/operator_splitting/coupling_or_godunov.tpp:12-131): per coupling
  step the fiber solver advances, its Vm is mapped onto the 3D mesh (slot 0 -> slot 0, the
  "connectedSlotsTerm1To2" {0: 0} of the example; mapping_between_meshes), then the bidomain solver runs.
* ``surface`` / ``sample`` -- the values OutputSurface takes: one face of the 3D mesh ("0-", "0+", "1-", ...)
  or interpolated at electrode positions.

Everything numeric runs in libfdm_b200.so (fdm_emg_* in include/fdm_b200.h): assembly of the stiffness
stencils, the potential flow and its gradient field, the fiber -> mesh transfer straight from the fiber
solver's device Vm, and the conjugate-gradient solve.  Settings keys read (reference names): StaticBidomainSolver
``timeStepWidth``, ``solverName``, ``initialGuessNonzero``; ``PotentialFlow``/``Activation`` ->
``FiniteElementMethod`` ``meshName``, ``prefactor``, ``dirichletBoundaryConditions``, ``diffusionTensor``,
``extracellularDiffusionTensor``; ``Solvers`` entries ``relativeTolerance``, ``absoluteTolerance``,
``maxIterations``; ``Meshes`` 3D entries with ``nElements`` and ``physicalExtent``/``physicalOffset`` or
``nodePositions``; ``MappingsBetweenMeshes`` ``xiTolerance``, ``defaultValue``; Coupling ``timeStepWidth``,
``endTime``, ``connectedSlotsTerm1To2``.  The linear solver is conjugate gradients with a Jacobi
or geometric-multigrid preconditioner whatever ``solverType`` names (both systems are symmetric positive
(semi)definite): ``preconditionerType`` "gamg", "mg", "hypre"/"boomeramg" select the multigrid V-cycle, any
other name the Jacobi preconditioner, none given the V-cycle from 300,000 nodes and Jacobi below (the
potential flow always uses Jacobi); quadrature: Gauss 3 points per direction for the potential flow and 5 for the activation
(the template arguments of fast_fibers_emg.cpp), changeable with a "B200" dict (``gaussPointsPotentialFlow``,
``gaussPointsActivation``).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Callable, Dict, Optional, Sequence

import numpy as np

from . import _native as N
from . import solver as S

# mesh size from which the multigrid preconditioner is the default
MULTIGRID_MIN_NODES = 300_000
# PETSc's defaults where a solver entry leaves a key out
_SOLVER_DEFAULTS = {"relativeTolerance": 1e-5, "absoluteTolerance": 1e-50, "maxIterations": 10000}
FACES = {"0-": (0, 0), "0+": (0, 1), "1-": (1, 0), "1+": (1, 1), "2-": (2, 0), "2+": (2, 1)}


def mesh_from_settings(mesh: dict):
    """(shape (nx, ny, nz) in nodes, node positions [N, 3]) of a structured 3D mesh entry."""
    ne = [int(x) for x in S._as_list(mesh["nElements"])]
    if len(ne) != 3:
        raise ValueError("settings: the 3D mesh needs three nElements")
    shape = (ne[0] + 1, ne[1] + 1, ne[2] + 1)
    if "nodePositions" in mesh:
        pos = np.asarray(mesh["nodePositions"], np.float64).reshape(-1, 3)
        if len(pos) != shape[0] * shape[1] * shape[2]:
            raise ValueError("settings: nodePositions does not match nElements")
        return shape, pos
    ext = [float(x) for x in S._as_list(mesh.get("physicalExtent", ne))]
    off = [float(x) for x in S._as_list(mesh.get("physicalOffset", [0.0, 0.0, 0.0]))]
    xs = [off[d] + np.linspace(0.0, ext[d], shape[d]) for d in range(3)]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    return shape, np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def fiber_positions_from_settings(meshes: dict, names: Sequence[str]) -> np.ndarray:
    """Node positions [n_nodes, 3] of the fibers in the fiber solver's node order: ``nodePositions``, or a
    1D mesh along x from ``physicalOffset``."""
    out = []
    for name in names:
        m = meshes[name]
        if "nodePositions" in m:
            out.append(np.asarray(m["nodePositions"], np.float64).reshape(-1, 3))
        else:
            n = int(S._as_list(m["nElements"])[0])
            L = float(S._as_list(m.get("physicalExtent", [n]))[0])
            off = np.zeros(3)
            o = S._as_list(m.get("physicalOffset", []))
            off[:len(o)] = o
            p = np.zeros((n + 1, 3)) + off
            p[:, 0] += np.linspace(0.0, L, n + 1)
            out.append(p)
    return np.concatenate(out) if out else np.zeros((0, 3))


def _tensors(v, n_elements: int) -> np.ndarray:
    """"diffusionTensor" entries: one 9-value list for all elements or one per element."""
    t = np.asarray(v if v is not None else np.eye(3).ravel(), np.float64)
    t = t.reshape(-1, 9)
    if len(t) not in (1, n_elements):
        raise ValueError("settings: one diffusion tensor for all elements or one per element")
    return np.ascontiguousarray(t)


def _dirichlet(bc, n_nodes: int):
    """{node: value} with negative node numbers counted from the end."""
    if not bc:
        return np.zeros(0, np.int64), np.zeros(0)
    items = bc.items() if isinstance(bc, dict) else enumerate(bc)
    nodes, vals = [], []
    for k, v in items:
        if v is None:
            continue
        k = int(k)
        nodes.append(k + n_nodes if k < 0 else k)
        vals.append(float(v[0] if isinstance(v, (list, tuple)) else v))
    return np.asarray(nodes, np.int64), np.asarray(vals)


class StaticBidomainSolver:
    """TimeSteppingScheme::StaticBidomainSolver on the device (reference method names)."""

    def __init__(self, shape, node_positions, sigma_i, sigma_e, *, dirichlet_nodes=None, dirichlet_values=None,
                 direction=None, potential_flow_solver: Optional[dict] = None,
                 emg_solver: Optional[dict] = None, initial_guess_nonzero: bool = True,
                 gauss_points_potential_flow: int = 3, gauss_points_activation: int = 5, device: int = 0,
                 preconditioner: Optional[str] = None):
        self.shape = tuple(int(x) for x in shape)
        self.node_positions = np.ascontiguousarray(node_positions, np.float64).reshape(-1, 3)
        self.n_nodes = self.shape[0] * self.shape[1] * self.shape[2]
        self.n_elements = (self.shape[0] - 1) * (self.shape[1] - 1) * (self.shape[2] - 1)
        if len(self.node_positions) != self.n_nodes:
            raise ValueError("node_positions must hold nx*ny*nz nodes")
        self.sigma_i = _tensors(sigma_i, self.n_elements)
        self.sigma_e = _tensors(sigma_e, self.n_elements)
        self.dirichlet_nodes = None if dirichlet_nodes is None else np.asarray(dirichlet_nodes, np.int64)
        self.dirichlet_values = None if dirichlet_values is None else np.asarray(dirichlet_values, np.float64)
        self.direction = None if direction is None else np.ascontiguousarray(direction, np.float64).reshape(-1, 3)
        if self.direction is None and (self.dirichlet_nodes is None or len(self.dirichlet_nodes) == 0):
            raise ValueError("the potential flow needs Dirichlet boundary conditions (or give the directions)")
        self.pf_solver = {**_SOLVER_DEFAULTS, **(potential_flow_solver or {})}
        self.emg_solver = {**_SOLVER_DEFAULTS, **(emg_solver or {})}
        self.initial_guess_nonzero = bool(initial_guess_nonzero)
        self.gauss_pf = int(gauss_points_potential_flow)
        self.gauss_act = int(gauss_points_activation)
        self.device = int(device)
        name = (preconditioner or self.emg_solver.get("preconditionerType") or "auto").lower()
        if name == "auto":
            # the V-cycle's launches cost more than its saved iterations below a few hundred thousand nodes
            name = "multigrid" if self.n_nodes >= MULTIGRID_MIN_NODES else "jacobi"
        self.preconditioner = "multigrid" if name in ("multigrid", "gamg", "mg", "hypre", "boomeramg", "ml") \
            else "jacobi"
        self.multigrid_levels = 0
        self.start_time = 0.0
        self.end_time = 0.0
        self.potential_flow_iterations = 0
        self._h = None
        self.initialized = False

    @classmethod
    def from_settings(cls, config: dict, meshes: dict, solvers: Optional[dict] = None, **kw):
        """From a "StaticBidomainSolver" settings dict plus the "Meshes" and "Solvers" dicts."""
        sb = config.get("StaticBidomainSolver", config)
        pf = sb["PotentialFlow"]["FiniteElementMethod"]
        act = sb["Activation"]["FiniteElementMethod"]
        shape, pos = mesh_from_settings(meshes[act["meshName"]])
        nodes, vals = _dirichlet(pf.get("dirichletBoundaryConditions"), len(pos))
        solvers = solvers or {}
        b200 = sb.get("B200", {})
        n_el = (shape[0] - 1) * (shape[1] - 1) * (shape[2] - 1)
        pre = float(act.get("prefactor", 1.0))
        return cls(shape, pos, _tensors(act.get("diffusionTensor"), n_el) * pre,
                   _tensors(act.get("extracellularDiffusionTensor"), n_el) * pre,
                   dirichlet_nodes=nodes, dirichlet_values=vals,
                   potential_flow_solver=solvers.get(pf.get("solverName", ""), {}),
                   emg_solver=solvers.get(sb.get("solverName", act.get("solverName", "")), {}),
                   initial_guess_nonzero=sb.get("initialGuessNonzero", True),
                   gauss_points_potential_flow=int(b200.get("gaussPointsPotentialFlow", 3)),
                   gauss_points_activation=int(b200.get("gaussPointsActivation", 5)), **kw)

    # -- lifecycle ------------------------------------------------------------------------------
    def _call(self, f, *args):
        rc = f(self._h, *args)
        if rc != N.FDM_OK:
            msg = N.lib().fdm_emg_last_error(self._h)
            raise N.FdmError(rc, msg.decode() if msg else "")

    def initialize(self):
        if self.initialized:
            return
        L = N.lib()
        h = C.c_void_p()
        nx, ny, nz = self.shape
        rc = L.fdm_emg_create(nx, ny, nz, N.ptr(self.node_positions, C.c_double), self.device, C.byref(h))
        if rc != N.FDM_OK:
            msg = L.fdm_emg_last_error(None)
            raise N.FdmError(rc, msg.decode() if msg else "")
        self._h = h
        try:
            if self.direction is not None:
                self._call(L.fdm_emg_set_direction, N.ptr(self.direction, C.c_double))
            else:
                its = C.c_int()
                self._call(L.fdm_emg_potential_flow, len(self.dirichlet_nodes),
                           N.ptr(np.ascontiguousarray(self.dirichlet_nodes), C.c_int64),
                           N.ptr(np.ascontiguousarray(self.dirichlet_values), C.c_double), self.gauss_pf,
                           float(self.pf_solver["relativeTolerance"]), float(self.pf_solver["absoluteTolerance"]),
                           int(self.pf_solver["maxIterations"]), C.byref(its))
                self.potential_flow_iterations = its.value
            self._call(L.fdm_emg_set_conductivity, len(self.sigma_i), N.ptr(self.sigma_i, C.c_double),
                       len(self.sigma_e), N.ptr(self.sigma_e, C.c_double), self.gauss_act)
            lv = C.c_int()
            self._call(L.fdm_emg_set_preconditioner, N.EMG_PRECOND_MULTIGRID if self.preconditioner == "multigrid"
                       else N.EMG_PRECOND_JACOBI, C.byref(lv))
            self.multigrid_levels = lv.value
        except Exception:
            self.close()
            raise
        self.initialized = True

    def close(self):
        if self._h is not None:
            N.lib().fdm_emg_destroy(self._h)
            self._h = None
        self.initialized = False

    def __enter__(self):
        self.initialize()
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference API ---------------------------------------------------------------------------
    def setTimeSpan(self, start_time: float, end_time: float):
        self.start_time, self.end_time = float(start_time), float(end_time)

    def advanceTimeSpan(self):
        """One static solve with the current Vm on the 3D mesh (static_bidomain_solver.tpp:37-55)."""
        self.initialize()
        its, res = C.c_int(), C.c_double()
        self._call(N.lib().fdm_emg_solve, float(self.emg_solver["relativeTolerance"]),
                   float(self.emg_solver["absoluteTolerance"]), int(self.emg_solver["maxIterations"]),
                   int(self.initial_guess_nonzero), C.byref(its), C.byref(res))
        return its.value

    def run(self):
        self.initialize()
        self.advanceTimeSpan()

    # -- transfer in --------------------------------------------------------------------------------
    def set_fiber_mapping(self, fiber_positions, xi_tolerance: float = 0.1, default_value: float = 0.0) -> int:
        """Fiber node positions [n, 3] in the fiber solver's node order; returns how many lie in the mesh."""
        self.initialize()
        p = np.ascontiguousarray(fiber_positions, np.float64).reshape(-1, 3)
        n = C.c_int64()
        self._call(N.lib().fdm_emg_set_fiber_mapping, len(p), N.ptr(p, C.c_double), float(xi_tolerance),
                   float(default_value), C.byref(n))
        return n.value

    def map_fibers(self, fiber_solver: S.FastMonodomainSolver):
        """Vm of the fiber solver (device to device, ordered after its advance) onto the 3D mesh."""
        self._call(N.lib().fdm_emg_map_fibers, fiber_solver._h)

    def map_values(self, fiber_values):
        v = np.ascontiguousarray(fiber_values, np.float64)
        self._call(N.lib().fdm_emg_map_values, N.ptr(v, C.c_double))

    def set_vm(self, vm):
        self.initialize()
        v = np.ascontiguousarray(vm, np.float64)
        if v.shape != (self.n_nodes,):
            raise ValueError("vm must hold one value per 3D node")
        self._call(N.lib().fdm_emg_set_vm, N.ptr(v, C.c_double))

    # -- results ---------------------------------------------------------------------------------
    def _get(self, field: int, n: int) -> np.ndarray:
        out = np.empty(n)
        self._call(N.lib().fdm_emg_get, field, N.ptr(out, C.c_double))
        return out

    def phi_e(self) -> np.ndarray:
        return self._get(N.EMG_PHI_E, self.n_nodes)

    def vm(self) -> np.ndarray:
        return self._get(N.EMG_VM, self.n_nodes)

    def rhs(self) -> np.ndarray:
        return self._get(N.EMG_RHS, self.n_nodes)

    def flow_potential(self) -> np.ndarray:
        return self._get(N.EMG_FLOW_POTENTIAL, self.n_nodes)

    def fiber_direction(self) -> np.ndarray:
        return self._get(N.EMG_DIRECTION, 3 * self.n_nodes).reshape(-1, 3)

    def stencil(self, which: int = 1) -> np.ndarray:
        """The assembled 27-point stencil [27, N] of K(sigma_i) (0) or K(sigma_i + sigma_e) (1)."""
        out = np.empty(27 * self.n_nodes)
        self._call(N.lib().fdm_emg_get_stencil, which, N.ptr(out, C.c_double))
        return out.reshape(27, self.n_nodes)

    def timing(self) -> Dict[str, float]:
        ms, its, res = C.c_double(), C.c_int(), C.c_double()
        N.lib().fdm_emg_timing(self._h, C.byref(ms), C.byref(its), C.byref(res))
        return {"solve_ms": ms.value, "iterations": its.value, "residual": res.value}

    def data(self) -> Dict[str, np.ndarray]:
        """The bidomain solver's field variables (static_bidomain.h: flowPotential, fiberDirection,
        transmembranePotential, transmembraneFlow, extraCellularPotential)."""
        return {"flowPotential": self.flow_potential(), "fiberDirection": self.fiber_direction(),
                "transmembranePotential": self.vm(), "transmembraneFlow": self.rhs(),
                "extraCellularPotential": self.phi_e()}

    def surface(self, face: str = "0+", values: Optional[np.ndarray] = None) -> np.ndarray:
        """phi_e (or ``values``) on one face of the mesh ("0-" x-min ... "2+" z-max) as a 2D array indexed by
        the two remaining directions (slowest first), the data OutputSurface writes."""
        axis, side = FACES[face]
        v = (self.phi_e() if values is None else np.asarray(values)).reshape(self.shape[::-1])  # [z, y, x]
        idx = [slice(None)] * 3
        idx[2 - axis] = -1 if side else 0
        return v[tuple(idx)]

    def sample(self, points, values: Optional[np.ndarray] = None) -> np.ndarray:
        """phi_e (or ``values``) interpolated at points [k, 3] (electrodes) with the trilinear shape functions of
        the element holding each point (NaN outside the mesh)."""
        v = self.phi_e() if values is None else np.asarray(values)
        pts = np.asarray(points, np.float64).reshape(-1, 3)
        nx, ny, nz = self.shape
        pos = self.node_positions
        out = np.full(len(pts), np.nan)
        for k, x in enumerate(pts):
            found = _find_element(pos, self.shape, x)
            if found is None:
                continue
            nodes, xi = found
            phi = _shape(xi)
            out[k] = phi @ v[nodes]
        return out


def _shape(xi):
    return np.array([(xi[0] if l & 1 else 1 - xi[0]) * (xi[1] if l & 2 else 1 - xi[1]) * (xi[2] if l & 4 else 1 - xi[2])
                     for l in range(8)])


def _find_element(pos, shape, x, tol: float = 1e-9):
    """(element node numbers, xi) of the element holding x, by bounding boxes and Newton's method."""
    nx, ny, nz = shape
    P = pos.reshape(nz, ny, nx, 3)
    lo = np.minimum.reduce([P[c:nz - 1 + c, b:ny - 1 + b, a:nx - 1 + a] for a in (0, 1) for b in (0, 1) for c in (0, 1)])
    hi = np.maximum.reduce([P[c:nz - 1 + c, b:ny - 1 + b, a:nx - 1 + a] for a in (0, 1) for b in (0, 1) for c in (0, 1)])
    cand = np.argwhere(np.all((x >= lo - tol) & (x <= hi + tol), axis=-1))
    for ez, ey, ex in cand:
        nodes = np.array([(ex + (l & 1)) + nx * ((ey + ((l >> 1) & 1)) + ny * (ez + (l >> 2))) for l in range(8)])
        Pe = pos[nodes]
        xi = np.full(3, 0.5)
        for _ in range(50):
            phi = _shape(xi)
            g = np.array([[(1 if l & 1 else -1) * (xi[1] if l & 2 else 1 - xi[1]) * (xi[2] if l & 4 else 1 - xi[2]),
                           (xi[0] if l & 1 else 1 - xi[0]) * (1 if l & 2 else -1) * (xi[2] if l & 4 else 1 - xi[2]),
                           (xi[0] if l & 1 else 1 - xi[0]) * (xi[1] if l & 2 else 1 - xi[1]) * (1 if l & 4 else -1)]
                          for l in range(8)])
            dx = np.linalg.solve(Pe.T @ g, phi @ Pe - x)
            xi -= dx
            if np.max(np.abs(dx)) < 1e-15:
                break
        if np.all(xi >= -1e-9) and np.all(xi <= 1 + 1e-9):
            return nodes, xi
    return None


class Coupling:
    """Control::Coupling of the fiber solver (Term1) and the static bidomain solver (Term2): per step of
    ``time_step_width`` the fibers advance, their Vm is mapped onto the 3D mesh and phi_e is solved
    (coupling_or_godunov.tpp:12-131); ``callback(step, t, bidomain)`` runs after each step's solve.

    Nothing flows back from the bidomain solver to the fibers (connectedSlotsTerm2To1 [None]), so with
    ``overlap`` (default) the solve of step k runs on its own stream, driven by a worker thread, while the
    fibers advance step k + 1; the transfer of step k + 1 waits for that solve.  The results are those of the
    sequential order."""

    def __init__(self, term1: S.FastMonodomainSolver, term2: StaticBidomainSolver, time_step_width: float,
                 end_time: float, fiber_positions, start_time: float = 0.0, xi_tolerance: float = 0.1,
                 default_value: float = 0.0, callback: Optional[Callable] = None, overlap: bool = True):
        self.term1, self.term2 = term1, term2
        self.time_step_width = float(time_step_width)
        self.start_time, self.end_time = float(start_time), float(end_time)
        self.fiber_positions = np.ascontiguousarray(fiber_positions, np.float64).reshape(-1, 3)
        if len(self.fiber_positions) != term1.system.n_nodes:
            raise ValueError("one position per fiber node needed")
        self.xi_tolerance, self.default_value = float(xi_tolerance), float(default_value)
        self.callback = callback
        self.overlap = bool(overlap)
        self.n_mapped = 0
        self.initialized = False
        self._pool = None

    @classmethod
    def from_settings(cls, config: dict, device: int = 0, **kw) -> "Coupling":
        """From a reference settings dict with a top-level "Coupling" (Term1: the FastMonodomainSolver's
        MultipleInstances, Term2: StaticBidomainSolver), "Meshes", "Solvers" and "MappingsBetweenMeshes"."""
        cp = config["Coupling"]
        slots = cp.get("connectedSlotsTerm1To2", {0: 0})
        pairs = list(slots.items()) if isinstance(slots, dict) else [(i, v) for i, v in enumerate(slots)]
        if [(int(a), int(b)) for a, b in pairs if b is not None] != [(0, 0)]:
            raise ValueError("settings: only the transfer of Vm (connectedSlotsTerm1To2 {0: 0}) is built")
        dt = float(cp.get("timeStepWidth", 1.0))
        end = float(cp.get("endTime", 1.0))
        term1 = dict(cp["Term1"])
        term1.setdefault("timeStepWidth", dt)
        term1.setdefault("endTime", end)
        fiber_cfg = {"Meshes": config.get("Meshes", {}), "RepeatedCall": term1}
        system = S.parse_settings(fiber_cfg, kw.pop("base_dir", "."))
        fibers = S.FastMonodomainSolver(system, device=device, **kw)
        meshes = config.get("Meshes", {})
        positions = fiber_positions_from_settings(meshes, system.fiber_mesh_names)
        emg = StaticBidomainSolver.from_settings(cp["Term2"], meshes, config.get("Solvers", {}), device=device)
        maps = config.get("MappingsBetweenMeshes", {})
        tol, default = 0.1, 0.0
        for name in system.fiber_mesh_names[:1]:
            entry = maps.get(name)
            targets = entry if isinstance(entry, list) else [entry]
            for t in targets:
                if isinstance(t, dict):
                    tol = float(t.get("xiTolerance", tol))
                    default = float(t.get("defaultValue", default))
        return cls(fibers, emg, dt, end, positions, start_time=float(cp.get("startTime", 0.0)), xi_tolerance=tol,
                   default_value=default)

    def initialize(self):
        if self.initialized:
            return
        self.term1.initialize()
        self.term2.initialize()
        self.n_mapped = self.term2.set_fiber_mapping(self.fiber_positions, self.xi_tolerance, self.default_value)
        self.initialized = True

    def n_time_steps(self) -> int:
        """TimeSteppingScheme::setTimeStepWidth (00_time_stepping_scheme.cpp:15-35)."""
        return max(1, int(math.ceil((self.end_time - self.start_time) / self.time_step_width - 0.1)))

    def advanceTimeSpan(self):
        self.initialize()
        n = self.n_time_steps()
        span = self.end_time - self.start_time
        dt = span / n
        t = self.start_time
        pending = None      # (future, step, time) of the solve still running

        def finish(p):
            p[0].result()
            if self.callback is not None:
                self.callback(p[1], p[2], self.term2)

        if self.overlap and self._pool is None:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=1, thread_name_prefix="bidomain")
        try:
            for k in range(n):
                self.term1.setTimeSpan(t, t + dt)
                self.term1.advanceTimeSpan()
                if pending is not None:
                    finish(pending)     # the previous solve reads the 3D Vm the transfer overwrites
                    pending = None
                self.term2.map_fibers(self.term1)
                self.term2.setTimeSpan(t, t + dt)
                if self.overlap:
                    pending = (self._pool.submit(self.term2.advanceTimeSpan), k, t + dt)
                else:
                    self.term2.advanceTimeSpan()
                    if self.callback is not None:
                        self.callback(k, t + dt, self.term2)
                t = self.start_time + (k + 1) / n * span
        finally:
            if pending is not None:
                finish(pending)

    def run(self):
        self.initialize()
        self.advanceTimeSpan()

    def close(self):
        if self._pool is not None:
            self._pool.shutdown(wait=True)
            self._pool = None
        self.term1.close()
        self.term2.close()

    def __enter__(self):
        self.initialize()
        return self

    def __exit__(self, *exc):
        self.close()
