"""Python settings harness and host-side operator API of the B200 FastMonodomainSolver.

:class:`FastMonodomainSolver` mirrors the reference class
``FastMonodomainSolverBase`` (core/src/specialized_solver/fast_monodomain_solver/
fast_monodomain_solver_base.h:85-124): ``initialize``, ``run``, ``advanceTimeSpan``,
``setTimeSpan``, ``startTime``, ``endTime``, ``data``, ``reset``,
``saveFiberDataCheckpoint`` and ``restoreFiberDataCheckpoint``, wrapped by the
RepeatedCall driver semantics (repeated_call.tpp:43-80).  It is constructed either from a
reference-style settings dict (:meth:`FastMonodomainSolver.from_settings`, the keys listed in
:func:`parse_settings`) or from a :class:`FiberSystem` of plain arrays.  All computation goes
through the C ABI of libfdm_b200.so; there is no CPU path.
"""
from __future__ import annotations

import copy
import ctypes as C
import math
import os
import warnings
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _native as N
from . import cellml as CM
from . import inputs
from . import models as MD
from . import output

SCHEMES = {"ImplicitEuler": 0, "CrankNicolson": 1}
METHODS = {"split": 0, "fused": 1}
PRECISIONS = {"fp64": 0, "fp32": 1}
CLAMP_RULES = {"vc": 0, "center": 1}
STIMULUS_MODES = {"clamp": 0, "current": 1}

#: parameter variants built into the library (see opendihu_b200/cellml.py VARIANTS)
VARIANT_PARAMETERS = {
    "hodgkin_huxley_1952": ((), (2, 3, 4)),
    "shorten_ocallaghan_davidson_soboleva_2007": ((32,), (65,)),
}


@dataclass
class FiberSystem:
    """Everything the solver needs, as arrays (node order = fibers concatenated)."""
    model: str
    fiber_offsets: np.ndarray                 # int64 [n_fibers+1]
    element_lengths: np.ndarray               # float64 [n_nodes - n_fibers]
    prefactor: np.ndarray                     # float64 [n_fibers]
    firing_events: np.ndarray                 # uint8 [rows, cols]
    motor_unit_no: np.ndarray                 # int32 [n_fibers]
    stimulation_point_index: np.ndarray       # int32 [n_fibers]
    call_frequency: np.ndarray                # float64 [n_fibers]
    repeat_after_first_call: np.ndarray       # float64 [n_fibers]
    call_enable_begin: np.ndarray             # float64 [n_fibers]
    jitter: np.ndarray = None                 # float64 [n_fibers, n_jitter]
    parameters: Optional[np.ndarray] = None   # float64 [n_params, n_nodes] (variant slots)
    states: Optional[np.ndarray] = None       # float64 [n_states, n_nodes]
    diffusion_scheme: str = "ImplicitEuler"
    dt_0d: float = 1e-4
    dt_1d: float = 1e-3
    dt_splitting: float = 1e-3
    dt_repeated_call: float = 1e-3
    start_time: float = 0.0
    end_time: float = 10.0
    approximate_exponential_function: bool = False
    value_for_stimulated_point: float = 20.0
    clamp_rule: str = "vc"
    vc_width: int = 4
    n_ranks: int = 1
    stimulus_mode: str = "clamp"
    stimulus_parameter: int = 0
    stimulus_value: float = 0.0
    algebraics_for_transfer: Sequence[int] = ()
    states_for_transfer: Sequence[int] = (0,)
    only_compute_if_has_been_stimulated: bool = False   # "onlyComputeIfHasBeenStimulated"
    skip_close_to_equilibrium: bool = False   # "disableComputationWhenStatesAreCloseToEquilibrium" (split, vc)
    # the diffusion solver has one more additional field variable than algebraicsForTransfer: the
    # "computeStateInformation" slot is transferred too (initialization.tpp:572-587)
    compute_state_information: bool = False
    # names of the fibers' meshes in the settings ("Meshes"), in fiber order (for their node positions)
    fiber_mesh_names: Sequence[str] = ()
    # "OutputWriter" entries of the diffusion solvers: (settings dict, fibers it covers); run after each
    # RepeatedCall piece of advanceTimeSpan (fast_monodomain_solver_compute.tpp:35-44)
    output_writers: Sequence = ()
    # "nAdditionalFieldVariables" of the diffusion solver: the output's additionalFieldVariable<k> fields
    n_additional_field_variables: int = 0
    # global fiber numbers ("additionalArgument" of the settings; default the fiber index), for the log
    fiber_numbers: Sequence[int] = ()
    # "stimulationLogFilename" of the CellML settings: the stimulation log written when the solver closes
    stimulation_log_filename: str = ""
    # "initializeStatesToEquilibrium" / "initializeStatesToEquilibriumTimestepWidth" of the CellML settings: the
    # initial states of every node are the equilibrium of the first node's initial states and parameters
    initialize_states_to_equilibrium: bool = False
    equilibrium_dt: float = 1e-4

    @property
    def n_fibers(self) -> int:
        return len(self.fiber_offsets) - 1

    @property
    def n_nodes(self) -> int:
        return int(self.fiber_offsets[-1])

    def copy(self) -> "FiberSystem":
        return copy.deepcopy(self)


def model_sizes(model: str):
    ns, na, npar, init, defaults = N.model_info(N.MODEL_IDS[model])
    return ns, na, npar, init, defaults


def uniform_fibers(model: str, lengths: Sequence[int], dx: float, prefactor, *, firing_events=None,
                   motor_unit_no=None, call_frequency: float = 0.1, repeat_after_first_call: float = 0.1,
                   call_enable_begin: float = 0.0, jitter=None, **kw) -> FiberSystem:
    """Straight fibers of the given node counts and element length dx (cm)."""
    lengths = np.asarray(lengths, np.int64)
    nf = len(lengths)
    off = np.zeros(nf + 1, np.int64)
    off[1:] = np.cumsum(lengths)
    elem = np.full(int(off[-1]) - nf, float(dx))
    pf = np.broadcast_to(np.asarray(prefactor, np.float64), (nf,)).copy()
    if firing_events is None:
        firing_events = np.ones((1, 1), np.uint8)
    if motor_unit_no is None:
        motor_unit_no = np.zeros(nf, np.int32)
    return FiberSystem(
        model=model, fiber_offsets=off, element_lengths=elem, prefactor=pf,
        firing_events=np.asarray(firing_events, np.uint8), motor_unit_no=np.asarray(motor_unit_no, np.int32),
        stimulation_point_index=(lengths // 2).astype(np.int32),
        call_frequency=np.full(nf, call_frequency), repeat_after_first_call=np.full(nf, repeat_after_first_call),
        call_enable_begin=np.full(nf, call_enable_begin),
        jitter=np.zeros((nf, 0)) if jitter is None else np.asarray(jitter, np.float64), **kw)


# ----------------------------------------------------------------------------------------------
# reference settings dict
# ----------------------------------------------------------------------------------------------

def _as_list(v):
    if v is None:
        return []
    if isinstance(v, (list, tuple, np.ndarray)):
        return list(v)
    return [v]


def _first_key(d: dict, *keys):
    for k in keys:
        if k in d:
            return k, d[k]
    return None, None


def _mesh_element_lengths(meshes: dict, name: str) -> np.ndarray:
    m = meshes[name]
    if "nodePositions" in m:
        p = np.asarray(m["nodePositions"], np.float64).reshape(-1, 3)
        return np.sqrt(np.sum((p[1:] - p[:-1]) ** 2, axis=1))
    n = int(_as_list(m["nElements"])[0])
    L = float(_as_list(m.get("physicalExtent", [n]))[0])
    return np.full(n, L / n)


def parse_settings(config: dict, base_dir: str = ".") -> FiberSystem:
    """Read a reference settings dict of ``RepeatedCall`` -> ``FastMonodomainSolver`` -> ``MultipleInstances``
    -> ``StrangSplitting`` -> (``Heun``/``CellML``, ``ImplicitEuler``|``CrankNicolson``/``FiniteElementMethod``).

    Keys read (with the reference defaults): RepeatedCall ``timeStepWidth``/``endTime``/``startTime``;
    FastMonodomainSolver ``fiberDistributionFile``, ``firingTimesFile``, ``valueForStimulatedPoint`` (20),
    ``neuromuscularJunctionRelativeSize`` (0), ``onlyComputeIfHasBeenStimulated``,
    ``disableComputationWhenStatesAreCloseToEquilibrium``, ``useSinglePrecision``; Strang ``timeStepWidth``;
    Heun ``timeStepWidth``; CellML ``modelFilename``, ``approximateExponentialFunction``,
    ``setSpecificStates{CallFrequency,FrequencyJitter,RepeatAfterFirstCall,CallEnableBegin}``,
    ``additionalArgument``, ``parametersUsedAsAlgebraic``, ``parametersUsedAsConstant``,
    ``parametersInitialValues``, ``statesInitialValues``, ``algebraicsForTransfer``, ``statesForTransfer``,
    ``mappings`` (instead of the four keys before it), ``stimulationLogFilename``; diffusion ``timeStepWidth``,
    ``nAdditionalFieldVariables``, ``OutputWriter``; FiniteElementMethod ``prefactor``, ``meshName``; ``Meshes``
    entries with ``nElements``/``physicalExtent`` or ``nodePositions``.  The code-generation keys
    (``generateGPUSource``, ``libraryFilename``, ``compilerFlags``, ``preCompileCommand``,
    ``postCompileCommand``, ``maximumNumberOfThreads``, ``useAoVSMemoryLayout``) are accepted and have no effect:
    the kernels are compiled into the library.  B200 options go in an optional ``"B200"`` dict
    next to the FastMonodomainSolver keys (``method``, ``precision``, ``clampRule``, ``vcWidth``,
    ``nRanks``, ``stimulusMode``, ``stimulusParameter``, ``stimulusValue``, ``neuromuscularJunctionSeed``).
    """
    key, rc = _first_key(config, "RepeatedCall")
    if rc is None:
        raise ValueError("settings: expected a top-level 'RepeatedCall' entry")
    fast = rc
    b200 = dict(fast.get("B200", {}))
    dt_rc = float(rc.get("timeStepWidth", 1e-3))
    end = float(rc.get("endTime", 1.0))
    start = float(rc.get("startTime", 0.0))
    meshes = config.get("Meshes", {})
    instances = fast["MultipleInstances"]["instances"]
    fibers: List[dict] = []
    writers = []
    for inst in instances:
        _, strang = _first_key(inst, "StrangSplitting", "Strang")
        if strang is None:
            raise ValueError("settings: every instance needs a 'StrangSplitting' entry")
        t1 = strang["Term1"]["MultipleInstances"]["instances"]
        t2 = strang["Term2"]["MultipleInstances"]["instances"]
        first = len(fibers)
        for a, b in zip(t1, t2):
            heun = a["Heun"]
            scheme, diff = _first_key(b, "ImplicitEuler", "CrankNicolson")
            if scheme is None:
                raise ValueError("settings: Timestepping scheme of diffusion in FastMonodomainSolver must be either "
                                 "ImplicitEuler or CrankNicolson")
            # a fiber's own diffusion writers
            writers += [(w, [len(fibers)]) for w in (diff.get("OutputWriter") or [])]
            fibers.append({"strang": strang, "heun": heun, "cellml": heun["CellML"], "scheme": scheme,
                           "diff": diff, "fem": diff["FiniteElementMethod"]})
        # the writers of the diffusion's MultipleInstances cover all its fibers
        writers += [(w, list(range(first, len(fibers))))
                    for w in (strang["Term2"]["MultipleInstances"].get("OutputWriter") or [])]
    if not fibers:
        raise ValueError("settings: no fibers")
    f0 = fibers[0]
    cellml = f0["cellml"]
    model_file = cellml["modelFilename"]
    if not os.path.isabs(model_file):
        model_file = os.path.join(base_dir, model_file)
    model = os.path.splitext(os.path.basename(model_file))[0]

    # geometry
    lengths = []
    elem = []
    for fb in fibers:
        name = fb["fem"].get("meshName", fb["cellml"].get("meshName"))
        h = _mesh_element_lengths(meshes, name)
        elem.append(h)
        lengths.append(len(h) + 1)
    lengths = np.asarray(lengths, np.int64)
    nf = len(lengths)
    off = np.zeros(nf + 1, np.int64)
    off[1:] = np.cumsum(lengths)
    prefactor = np.array([float(fb["fem"].get("prefactor", 1.0)) for fb in fibers])

    # parameters: map the settings' parameter list onto the built variant's slots
    if cellml.get("mappings"):
        # parameters and transfer slots by name (00_cellml_adapter_base.tpp:160-607); the key replaces
        # parametersUsedAs*, statesForTransfer and algebraicsForTransfer
        if model in VARIANT_PARAMETERS:
            names = CM.model_variable_names(model)
        elif os.path.exists(model_file):
            m = CM.parse_model_file(model_file)
            names = {"state": m.state_names, "algebraic": m.algebraic_names, "constant": m.constant_names}
        else:
            raise ValueError(f"settings: model file {model_file!r} not found")
        mp = CM.parse_mappings(cellml["mappings"], names)
        pa, pc = mp["parametersUsedAsAlgebraic"], mp["parametersUsedAsConstant"]
        st_transfer, alg_transfer = mp["statesForTransfer"], mp["algebraicsForTransfer"]
    else:
        pa = [int(x) for x in _as_list(cellml.get("parametersUsedAsAlgebraic", []))]
        pc = [int(x) for x in _as_list(cellml.get("parametersUsedAsConstant", []))]
        st_transfer = [int(x) for x in _as_list(cellml.get("statesForTransfer", [0]))]
        alg_transfer = [int(x) for x in _as_list(cellml.get("algebraicsForTransfer", []))]
    if model in VARIANT_PARAMETERS and MD.builtin_variant(model, pa, pc):
        pa_var, pc_var = VARIANT_PARAMETERS[model]
    else:
        # a variant (or model) the library does not carry: generated, compiled and loaded as a model module, as
        # the reference generates and compiles its model library at run time (gpu.tpp:106-205)
        model = MD.load_model(model, pa, pc, model_file=model_file if os.path.exists(model_file) else None)
        pa_var, pc_var = tuple(pa), tuple(pc)
    ns, na, npar, init, defaults = model_sizes(model)
    n_user = len(pa) + len(pc)
    slot_of = list(range(len(pa))) + [len(pa_var) + pc_var.index(c) for c in pc]
    n_nodes = int(off[-1])
    params = np.repeat(defaults[:, None], n_nodes, axis=1) if npar else np.zeros((0, n_nodes))
    for fi, fb in enumerate(fibers):
        vals = [float(x) for x in _as_list(fb["cellml"].get("parametersInitialValues", []))]
        n_here = int(lengths[fi])
        if len(vals) == n_user:
            for j in range(n_user):
                params[slot_of[j], off[fi]:off[fi + 1]] = vals[j]
        elif len(vals) == n_user * n_here and n_user > 0:
            arr = np.asarray(vals).reshape(n_here, n_user)
            for j in range(n_user):
                params[slot_of[j], off[fi]:off[fi + 1]] = arr[:, j]
        else:
            # the reference pads missing values with 0 (00_source_code_generator_base.cpp:67-81)
            padded = (vals + [0.0] * n_user)[:n_user]
            for j in range(n_user):
                params[slot_of[j], off[fi]:off[fi + 1]] = padded[j]

    states = None
    if "statesInitialValues" in cellml and _as_list(cellml["statesInitialValues"]):
        v = np.asarray(_as_list(cellml["statesInitialValues"]), np.float64)
        if len(v) == ns:
            states = np.repeat(v[:, None], n_nodes, axis=1)

    # stimulation inputs
    fdf = fast.get("fiberDistributionFile", "")
    ftf = fast.get("firingTimesFile", "")
    mus = inputs.parse_fiber_distribution(open(os.path.join(base_dir, fdf)).read()) if fdf else [0]
    rows = inputs.parse_firing_times(open(os.path.join(base_dir, ftf)).read()) if ftf else [[0]]
    firing = inputs.firing_matrix(rows)
    mu_no = np.zeros(nf, np.int32)
    freq = np.zeros(nf)
    rep = np.zeros(nf)
    beg = np.zeros(nf)
    jit_lists = []
    fiber_numbers = []
    for fi, fb in enumerate(fibers):
        c = fb["cellml"]
        fiber_no_global = int(c.get("additionalArgument", fi)) if isinstance(c.get("additionalArgument", fi), (int, np.integer)) else fi
        mu_no[fi] = mus[fiber_no_global % len(mus)]
        fiber_numbers.append(fiber_no_global)
        freq[fi] = float(c.get("setSpecificStatesCallFrequency", 0.0) or 0.0)
        rep[fi] = float(c.get("setSpecificStatesRepeatAfterFirstCall", 0.0) or 0.0)
        beg[fi] = float(c.get("setSpecificStatesCallEnableBegin", 0.0) or 0.0)
        jit_lists.append([float(x) for x in _as_list(c.get("setSpecificStatesFrequencyJitter", []))])
    nj = max(len(j) for j in jit_lists)
    if any(len(j) != nj for j in jit_lists):
        raise ValueError("settings: all fibers need the same number of setSpecificStatesFrequencyJitter values")
    jitter = np.asarray(jit_lists, np.float64).reshape(nf, nj)
    nmj_size = float(fast.get("neuromuscularJunctionRelativeSize", 0.0))
    if nmj_size <= 0:
        center = (lengths // 2).astype(np.int32)
    else:
        rng = np.random.default_rng(int(b200.get("neuromuscularJunctionSeed", 0)))
        u = rng.uniform(0.5 - nmj_size / 2, 0.5 + nmj_size / 2, size=nf)
        center = (lengths * u).astype(np.int32)
    # both options default to True in the reference (fast_monodomain_solver_initialization.tpp:68-69); its
    # "gpu" optimizationType ignores them (fast_monodomain_solver_gpu.tpp computes every node)
    vc_path = cellml.get("optimizationType", "vc") == "vc"
    only_if_stimulated = vc_path and bool(fast.get("onlyComputeIfHasBeenStimulated", True))
    skip_equilibrium = vc_path and bool(fast.get("disableComputationWhenStatesAreCloseToEquilibrium", True))

    precision = b200.get("precision", "fp32" if fast.get("useSinglePrecision", False) else "fp64")
    sys_ = FiberSystem(
        model=model, fiber_offsets=off, element_lengths=np.concatenate(elem), prefactor=prefactor,
        firing_events=firing, motor_unit_no=mu_no, stimulation_point_index=center, call_frequency=freq,
        repeat_after_first_call=rep, call_enable_begin=beg, jitter=jitter, parameters=params, states=states,
        diffusion_scheme=f0["scheme"], dt_0d=float(f0["heun"].get("timeStepWidth", 1e-4)),
        dt_1d=float(f0["diff"].get("timeStepWidth", 1e-3)), dt_splitting=float(f0["strang"].get("timeStepWidth", dt_rc)),
        dt_repeated_call=dt_rc, start_time=start, end_time=end,
        approximate_exponential_function=bool(cellml.get("approximateExponentialFunction",
                                                         cellml.get("optimizationType", "vc") == "vc")),
        value_for_stimulated_point=float(fast.get("valueForStimulatedPoint", 20.0)),
        clamp_rule=b200.get("clampRule", "vc" if cellml.get("optimizationType", "vc") == "vc" else "center"),
        vc_width=int(b200.get("vcWidth", 4)), n_ranks=int(b200.get("nRanks", 1)),
        stimulus_mode=b200.get("stimulusMode", "clamp"), stimulus_parameter=int(b200.get("stimulusParameter", 0)),
        stimulus_value=float(b200.get("stimulusValue", 0.0)),
        algebraics_for_transfer=alg_transfer, states_for_transfer=st_transfer or [0],
        only_compute_if_has_been_stimulated=only_if_stimulated, skip_close_to_equilibrium=skip_equilibrium)
    sys_.fiber_mesh_names = [fb["fem"].get("meshName", fb["cellml"].get("meshName")) for fb in fibers]
    sys_.compute_state_information = \
        int(f0["diff"].get("nAdditionalFieldVariables", 0)) > len(sys_.algebraics_for_transfer)
    sys_.output_writers = writers
    sys_.fiber_numbers = fiber_numbers
    sys_.stimulation_log_filename = str(cellml.get("stimulationLogFilename") or "")
    sys_.initialize_states_to_equilibrium = bool(cellml.get("initializeStatesToEquilibrium", False))
    sys_.equilibrium_dt = float(cellml.get("initializeStatesToEquilibriumTimestepWidth", 1e-4))
    sys_.n_additional_field_variables = int(f0["diff"].get("nAdditionalFieldVariables", 0))
    sys_.method = b200.get("method", "split")
    sys_.precision = precision
    return sys_


def piece_end(start: float, end: float, k: int, n: int) -> float:
    """End of RepeatedCall piece k of n over [start, end] (the Strang span's endTime, the reference's
    currentTime_): start + k/n*span + span/n, as repeated_call.tpp:59-70 forms it."""
    span = end - start
    t = start if k == 0 else start + k / n * span
    return t + span / n


def output_writers(system: FiberSystem) -> list:
    """The settings' output writers of a system (output.OutputWriter, fibers named by their meshes)."""
    names = list(system.fiber_mesh_names)
    return [output.OutputWriter(w, fibers, [names[f] if f < len(names) and names[f] else f"MeshFiber_{f}"
                                            for f in fibers])
            for w, fibers in system.output_writers]


def write_due_output(solver, due, current_time: float) -> None:
    """The diffusion data of the fibers each due writer covers, read through the solver's vm(), algebraics()
    and compute_state_information(): geometry (cumulative element lengths along x), "solution" (Vm) and
    additionalFieldVariable<k> (algebraicsForTransfer, then the computeStateInformation slot;
    fast_monodomain_solver_communication.tpp:437-488)."""
    s = solver.system
    vm = solver.vm()
    extra = []
    if len(s.algebraics_for_transfer):
        extra += list(solver.algebraics())
    if s.compute_state_information:
        extra.append(solver.compute_state_information())
    n_add = max(int(s.n_additional_field_variables), len(extra))
    off = np.asarray(s.fiber_offsets, np.int64)
    elem = np.asarray(s.element_lengths)
    for w, name in due:
        dicts = []
        for f in w.fibers:
            a, b = int(off[f]), int(off[f + 1])
            x = np.concatenate([[0.0], np.cumsum(elem[a - f:b - f - 1])])
            geom = np.stack([x, np.zeros_like(x), np.zeros_like(x)], axis=1)
            add = {f"additionalFieldVariable{k}": (extra[k][a:b] if k < len(extra) else np.zeros(b - a))
                   for k in range(n_add)}
            dicts.append(output.fiber_dict({"0": vm[a:b]}, geom, 0, current_time, "solution", add))
        w.write(name, dicts)


def equilibrium_states(system: FiberSystem, device: int = 0) -> Dict[str, object]:
    """The CellmlAdapter's equilibrium search (03_cellml_adapter.tpp:445-515) for the first node: its initial
    states (the settings' statesInitialValues or the model's) and parameters, RK4 with the settings' time step
    width (fdm_model_equilibrium).  A search that does not converge warns, as the reference logs an error, and
    returns its last values."""
    ns, _, npar, init, _ = model_sizes(system.model)
    y = np.ascontiguousarray(system.states[:, 0] if system.states is not None else init, np.float64).copy()
    p = np.ascontiguousarray(system.parameters[:, 0] if system.parameters is not None and npar else np.zeros(1),
                             np.float64)
    it, inc, dt = C.c_int64(), C.c_double(), C.c_double()
    N.check(N.lib().fdm_model_equilibrium(N.MODEL_IDS[system.model], int(device),
                                          int(bool(system.approximate_exponential_function)), N.ptr(p, C.c_double),
                                          float(system.equilibrium_dt), N.ptr(y, C.c_double), C.byref(it),
                                          C.byref(inc), C.byref(dt)))
    if not inc.value < 1e-5:
        warnings.warn(f"equilibrium values for the states were not found within {it.value} RK-4 steps: last "
                      f"increment {inc.value}, time step width {dt.value}")
    return {"states": y, "iterations": it.value, "max_increment": inc.value, "dt": dt.value}


def write_host_settings(system: FiberSystem, path: str, method: Optional[str] = None,
                        precision: Optional[str] = None, device: int = 0) -> None:
    """The parsed settings as the "key count value..." lines fdm::FiberSettings::load reads
    (include/fdm_b200.hpp): the input of the C++ host class fdm::FastMonodomainSolver."""
    s = system
    ns, _, npar, init, defaults = model_sizes(s.model)
    n = s.n_nodes
    states = s.states if s.states is not None else np.repeat(np.asarray(init)[:, None], n, axis=1)
    params = s.parameters if s.parameters is not None else np.repeat(np.asarray(defaults)[:, None], n, axis=1)
    fe = np.asarray(s.firing_events, np.uint8)
    jit = np.asarray(s.jitter if s.jitter is not None else np.zeros((s.n_fibers, 0)), np.float64)
    scalars = {
        "model": N.MODEL_IDS[s.model], "diffusion_scheme": SCHEMES[s.diffusion_scheme],
        "method": METHODS[method or getattr(s, "method", "split")],
        "reaction_precision": PRECISIONS[precision or getattr(s, "precision", "fp64")],
        "approximate_exponential_function": int(bool(s.approximate_exponential_function)),
        "clamp_rule": CLAMP_RULES[s.clamp_rule], "vc_width": s.vc_width, "n_ranks": s.n_ranks,
        "stimulus_mode": STIMULUS_MODES[s.stimulus_mode], "stimulus_parameter": s.stimulus_parameter,
        "stimulus_value": s.stimulus_value, "value_for_stimulated_point": s.value_for_stimulated_point,
        "dt_repeated_call": s.dt_repeated_call, "dt_splitting": s.dt_splitting, "dt_0d": s.dt_0d, "dt_1d": s.dt_1d,
        "only_compute_if_stimulated": int(bool(s.only_compute_if_has_been_stimulated)),
        "skip_close_to_equilibrium": int(bool(s.skip_close_to_equilibrium)), "device": device,
        "start_time": s.start_time, "end_time": s.end_time, "firing_rows": fe.shape[0], "firing_cols": fe.shape[1],
        "n_jitter": jit.shape[1] if jit.ndim == 2 else 0,
        "initialize_states_to_equilibrium": int(bool(s.initialize_states_to_equilibrium)),
        "equilibrium_dt": s.equilibrium_dt,
    }
    arrays = {
        "fiber_offsets": s.fiber_offsets, "element_lengths": s.element_lengths, "prefactor": s.prefactor,
        "parameters": params, "states": states, "firing_events": fe, "motor_unit_no": s.motor_unit_no,
        "stimulation_point_index": s.stimulation_point_index, "call_frequency": s.call_frequency,
        "repeat_after_first_call": s.repeat_after_first_call, "call_enable_begin": s.call_enable_begin,
        "jitter": jit, "algebraics_for_transfer": s.algebraics_for_transfer,
        "states_for_transfer": s.states_for_transfer,
        "fiber_numbers": s.fiber_numbers if len(s.fiber_numbers) == s.n_fibers else np.arange(s.n_fibers),
    }
    with open(path, "w") as f:
        f.write("# opendihu_b200 host settings: key count values\n")
        for k, v in scalars.items():
            f.write(f"{k} 1 {float(v)!r}\n")
        for k, v in arrays.items():
            a = np.asarray(v, np.float64).ravel()
            f.write(f"{k} {a.size} " + " ".join(repr(float(x)) for x in a) + "\n")


# ----------------------------------------------------------------------------------------------
# the operator
# ----------------------------------------------------------------------------------------------

class FastMonodomainSolver:
    """B200 FastMonodomainSolver (reference API names; see the module docstring)."""

    def __init__(self, system: FiberSystem, method: Optional[str] = None, precision: Optional[str] = None,
                 steps_per_launch: int = 0, threads_per_block: int = 0, nodes_per_thread: int = 0,
                 check_nan: bool = True, profile: bool = False, trace_nodes: Sequence[int] = (),
                 trace_capacity: int = 0, device: int = 0, autotune: bool = False, cluster_size: int = 0):
        self.system = system
        self.method = method or getattr(system, "method", "split")
        self.precision = precision or getattr(system, "precision", "fp64")
        self.steps_per_launch = steps_per_launch
        self.threads_per_block = threads_per_block
        self.nodes_per_thread = nodes_per_thread
        self.check_nan = check_nan
        self.profile = profile
        self.trace_nodes = np.asarray(trace_nodes, np.int64)
        self.trace_capacity = int(trace_capacity)
        self._act_cap = 0
        self.device = int(device)
        self.autotune = bool(autotune)
        #: fused method: CTAs of one thread-block cluster per fiber (0: chosen by the library, 1: off)
        self.cluster_size = int(cluster_size)
        self.tuning = None
        #: (first_node, count, evaluated) per fiber replacing the clamp selection of fdm_set_stimulation
        #: (set by the sharded solver to keep the selection of the unsharded layout)
        self.clamp_override = None
        #: per-node onlyComputeIfHasBeenStimulated codes replacing the library's selection (sharded solver)
        self.gate_override = None
        self._h = None
        self._start = system.start_time
        self._end = system.end_time
        self._ck = None
        self._writers = None
        self._log_on = False
        self._equilibrium_done = False
        #: result of the "initializeStatesToEquilibrium" search (states, iterations, max_increment, dt)
        self.equilibrium = None
        # the reference's currentTime_ (end of the last RepeatedCall piece) and nTimeStepsSplitting_ (its
        # split steps), which callOutputWriter hands to the writers
        self._current_time = system.start_time
        self._piece_steps = 0
        self.initialized = False

    @classmethod
    def from_settings(cls, config: dict, base_dir: str = ".", **kw) -> "FastMonodomainSolver":
        return cls(parse_settings(config, base_dir), **kw)

    # -- lifecycle ------------------------------------------------------------------------------
    def initialize(self):
        if self.initialized:
            return
        s = self.system
        L = N.lib()
        if self.method == "auto":
            # the autotuner times the split method against every fused shape and keeps the fastest
            from .autotune import autotune
            self.tuning = autotune(s, self.precision, device=self.device, include_split=True)
            self.method = self.tuning["method"]
            if self.method == "split":
                self.steps_per_launch = self.steps_per_launch or int(self.tuning["steps_per_launch"] or 0)
            else:
                self.threads_per_block = self.tuning["threads"]
                self.nodes_per_thread = self.tuning["nodes_per_thread"]
                self.cluster_size = int(self.tuning.get("cluster_size", 1))
                if not self.steps_per_launch:
                    self.steps_per_launch = self.tuning["steps_per_launch"]
        elif self.autotune and self.method == "fused" and not self.threads_per_block:
            from .autotune import autotune
            self.tuning = autotune(s, self.precision, device=self.device)
            self.threads_per_block = self.tuning["threads"]
            self.nodes_per_thread = self.tuning["nodes_per_thread"]
            self.cluster_size = int(self.tuning.get("cluster_size", 1))
            if not self.steps_per_launch:
                self.steps_per_launch = self.tuning["steps_per_launch"]
        cfg = N.default_config()
        cfg.model = N.MODEL_IDS[s.model]
        cfg.diffusion_scheme = SCHEMES[s.diffusion_scheme]
        cfg.method = METHODS[self.method]
        cfg.reaction_precision = PRECISIONS[self.precision]
        cfg.approximate_exponential_function = int(bool(s.approximate_exponential_function))
        cfg.clamp_rule = CLAMP_RULES[s.clamp_rule]
        cfg.vc_width = int(s.vc_width)
        cfg.n_ranks = int(s.n_ranks)
        cfg.stimulus_mode = STIMULUS_MODES[s.stimulus_mode]
        cfg.stimulus_parameter = int(s.stimulus_parameter)
        cfg.stimulus_value = float(s.stimulus_value)
        cfg.value_for_stimulated_point = float(s.value_for_stimulated_point)
        cfg.dt_repeated_call = float(s.dt_repeated_call)
        cfg.dt_splitting = float(s.dt_splitting)
        cfg.dt_0d = float(s.dt_0d)
        cfg.dt_1d = float(s.dt_1d)
        cfg.steps_per_launch = int(self.steps_per_launch)
        cfg.threads_per_block = int(self.threads_per_block)
        cfg.nodes_per_thread = int(self.nodes_per_thread)
        cfg.check_nan = int(bool(self.check_nan))
        cfg.profile = int(bool(self.profile))
        cfg.device = self.device
        cfg.only_compute_if_stimulated = int(bool(s.only_compute_if_has_been_stimulated))
        cfg.skip_close_to_equilibrium = int(bool(s.skip_close_to_equilibrium))
        cfg.cluster_size = int(self.cluster_size)
        h = C.c_void_p()
        N.check(L.fdm_create(C.byref(cfg), C.byref(h)))
        self._h = h
        try:
            off = np.ascontiguousarray(s.fiber_offsets, np.int64)
            elem = np.ascontiguousarray(s.element_lengths, np.float64)
            pf = np.ascontiguousarray(s.prefactor, np.float64)
            self._call(L.fdm_set_fibers, len(off) - 1, N.ptr(off, C.c_int64), N.ptr(elem, C.c_double),
                       N.ptr(pf, C.c_double))
            if s.parameters is not None and s.parameters.size:
                p = np.ascontiguousarray(s.parameters, np.float64)
                self._call(L.fdm_set_parameters, N.ptr(p, C.c_double))
            if s.initialize_states_to_equilibrium and not self._equilibrium_done:
                self.equilibrium = equilibrium_states(s, self.device)
                s.states = np.repeat(self.equilibrium["states"][:, None], s.n_nodes, axis=1)
                self._equilibrium_done = True
            if s.states is not None:
                st = np.ascontiguousarray(s.states, np.float64)
                self._call(L.fdm_set_states, N.ptr(st, C.c_double))
            self._set_stimulation()
            if self.clamp_override is not None:
                first, cnt, ev = (np.ascontiguousarray(a, t) for a, t in
                                  zip(self.clamp_override, (np.int64, np.int32, np.uint8)))
                self._call(L.fdm_set_clamp_nodes, N.ptr(first, C.c_int64), N.ptr(cnt, C.c_int),
                           N.ptr(ev, C.c_uint8))
            if self.gate_override is not None and s.only_compute_if_has_been_stimulated:
                codes = np.ascontiguousarray(self.gate_override, np.int32)
                self._call(L.fdm_set_gate_codes, N.ptr(codes, C.c_int))
            if len(s.algebraics_for_transfer):
                idx = np.ascontiguousarray(s.algebraics_for_transfer, np.int32)
                self._call(L.fdm_set_algebraics_for_transfer, len(idx), N.ptr(idx, C.c_int))
            if len(self.trace_nodes):
                self._call(L.fdm_set_trace, len(self.trace_nodes), N.ptr(self.trace_nodes, C.c_int64),
                           self.trace_capacity)
            if s.stimulation_log_filename:
                self._log_on = True
                self._call(L.fdm_set_stimulation_log, self._log_bound(s.end_time - s.start_time))
        except Exception:
            self.close()
            raise
        self.initialized = True

    def _set_stimulation(self):
        s = self.system
        fe = np.ascontiguousarray(s.firing_events, np.uint8)
        mu = np.ascontiguousarray(s.motor_unit_no, np.int32)
        ce = np.ascontiguousarray(s.stimulation_point_index, np.int32)
        fr = np.ascontiguousarray(s.call_frequency, np.float64)
        rp = np.ascontiguousarray(s.repeat_after_first_call, np.float64)
        bg = np.ascontiguousarray(s.call_enable_begin, np.float64)
        jit = np.ascontiguousarray(s.jitter if s.jitter is not None else np.zeros((s.n_fibers, 0)), np.float64)
        nj = jit.shape[1] if jit.ndim == 2 else 0
        jp = jit if jit.size else np.zeros(1)
        self._keep = (fe, mu, ce, fr, rp, bg, jp)
        self._call(N.lib().fdm_set_stimulation, N.ptr(fe, C.c_uint8), fe.shape[0], fe.shape[1], N.ptr(mu, C.c_int),
                   N.ptr(ce, C.c_int), N.ptr(fr, C.c_double), N.ptr(rp, C.c_double), N.ptr(bg, C.c_double),
                   N.ptr(jp, C.c_double), nj)

    def _call(self, f, *args):
        N.check(f(self._h, *args), self._h)

    def close(self):
        if self._h is not None:
            try:
                if self.system.stimulation_log_filename and self._log_on:
                    # the reference writes its log at the end of the run (dihu_context.cpp:85-86)
                    self.writeStimulationLog()
            finally:
                N.lib().fdm_destroy(self._h)
                self._h = None
        self.initialized = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        self.initialize()
        return self

    def __exit__(self, *exc):
        self.close()

    # -- reference operator API -----------------------------------------------------------------
    def setTimeSpan(self, start_time: float, end_time: float):
        self._start = float(start_time)
        self._end = float(end_time)

    def startTime(self) -> float:
        return self._start

    def endTime(self) -> float:
        return self._end

    def advanceTimeSpan(self, withOutputWritersEnabled: bool = True):
        """RepeatedCall over [startTime, endTime] (each repeated call is one setTimeSpan+advanceTimeSpan of
        the reference solver).  With output writers in the settings (and enabled) they run after every
        RepeatedCall piece, as the reference's advanceTimeSpan calls them (fast_monodomain_solver_compute.tpp:
        35-44): the advance stops only after the pieces whose call writes a file, the steps stay those of
        one advance over the span."""
        self.initialize()
        writers = self._output_writers() if withOutputWritersEnabled else []
        L = N.lib()
        self._prepare_advance()
        n = C.c_int64()
        self._call(L.fdm_repeated_call_plan, self._start, self._end, C.byref(n), None)
        steps = np.zeros(max(n.value, 1), np.int32)
        if self.system.output_writers:   # the split steps per piece, for the writers' call counts
            self._call(L.fdm_repeated_call_plan, self._start, self._end, C.byref(n), N.ptr(steps, C.c_int))
        if not writers:
            self._call(L.fdm_advance, self._start, self._end)
            self._current_time = self._piece_end(n.value - 1, n.value)
            self._piece_steps = int(steps[n.value - 1])
            return
        done = 0
        for k in range(n.value):
            t = self._piece_end(k, n.value)
            due = [(w, name) for w in writers for name in [w.prepare(0, t, int(steps[k]))] if name]
            self._piece_steps = int(steps[k])
            self._current_time = t
            if due:
                self._call(L.fdm_advance_pieces, self._start, self._end, done, k + 1)
                done = k + 1
                self._write_output(due)
        if done < n.value:
            self._call(L.fdm_advance_pieces, self._start, self._end, done, n.value)

    def callOutputWriter(self, timeStepNo: int, currentTime: float, callCountIncrement: int = 1):
        """The reference's callOutputWriter (fast_monodomain_solver_base.tpp:7-24): when timeStepNo is a
        multiple of callCountIncrement, the diffusion writers are called as after a RepeatedCall piece, with
        the end time and split steps of the last piece (0 steps before the first advance: the call then
        counts as the initial-values call, which always writes).  currentTime is not used, as in the
        reference."""
        self.initialize()
        if int(timeStepNo) % int(callCountIncrement) != 0:
            return
        due = [(w, name) for w in self._output_writers()
               for name in [w.prepare(0, self._current_time, self._piece_steps)] if name]
        if due:
            self._write_output(due)

    # -- stimulation log ----------------------------------------------------------------------------
    def enable_stimulation_log(self, capacity: int = 0):
        """Records every stimulation begin from now on (the reference's StimulationLogging; see
        fdm_set_stimulation_log); the capacity grows before each advance to what its span can need."""
        self.initialize()
        self._log_on = True
        self._call(N.lib().fdm_set_stimulation_log,
                   max(int(capacity), self._log_bound(self.system.end_time - self.system.start_time)))

    def _log_bound(self, span: float) -> int:
        """Stimulation begins a span can hold: a fiber's machine checks at most once per 1/(f (1 + jitter))."""
        s = self.system
        f = np.asarray(s.call_frequency, np.float64)
        jit = np.asarray(s.jitter, np.float64) if s.jitter is not None and np.size(s.jitter) else np.zeros((len(f), 1))
        rate = f * (1.0 + np.max(np.abs(jit.reshape(len(f), -1)), axis=1, initial=0.0)) if len(f) else f
        return int(np.sum(np.ceil(max(span, 0.0) * rate) + 2)) + 16

    def _grow_stimulation_log(self, span: float):
        n = C.c_int64()
        self._call(N.lib().fdm_get_stimulation_log, C.byref(n), None, None)
        self._call(N.lib().fdm_set_stimulation_log, n.value + self._log_bound(span))

    def stimulation_log(self) -> Dict[str, np.ndarray]:
        """The recorded stimulation begins, in time order: "time", "fiber" (global fiber numbers), "motorUnit"."""
        self.initialize()
        n = C.c_int64()
        self._call(N.lib().fdm_get_stimulation_log, C.byref(n), None, None)
        t = np.zeros(max(n.value, 1))
        f = np.zeros(max(n.value, 1), np.int32)
        self._call(N.lib().fdm_get_stimulation_log, C.byref(n), N.ptr(t, C.c_double), N.ptr(f, C.c_int))
        k = n.value  # the library fails (FDM_ERR_ARG) rather than return an incomplete log
        t, f = t[:k], f[:k]
        order = np.lexsort((f, t))
        t, f = t[order], f[order]
        nums = np.asarray(self.system.fiber_numbers if len(self.system.fiber_numbers) == self.system.n_fibers
                          else np.arange(self.system.n_fibers), np.int64)
        return {"time": t, "fiber": nums[f] if k else f.astype(np.int64),
                "motorUnit": np.asarray(self.system.motor_unit_no, np.int64)[f] if k else f.astype(np.int64)}

    def writeStimulationLog(self, filename: Optional[str] = None) -> str:
        """Writes the log in the reference's format (output.write_stimulation_log); the file name defaults to
        the settings' stimulationLogFilename."""
        name = filename or self.system.stimulation_log_filename
        if not name:
            raise ValueError("writeStimulationLog: no file name (settings have no stimulationLogFilename)")
        d = self.stimulation_log()
        output.write_stimulation_log(name, d["time"], d["fiber"], d["motorUnit"])
        return name

    def _piece_end(self, k: int, n: int) -> float:
        return piece_end(self._start, self._end, k, n)

    def _output_writers(self):
        if self._writers is None:
            self._writers = output_writers(self.system)
        return self._writers

    def _write_output(self, due):
        write_due_output(self, due, self._current_time)

    def _prepare_advance(self):
        """What an advance over [startTime, endTime] needs first: room in the stimulation log."""
        if self._log_on:
            self._grow_stimulation_log(self._end - self._start)

    def _advance_pieces(self, k_begin: int, k_end: int):
        self._call(N.lib().fdm_advance_pieces, self._start, self._end, k_begin, k_end)

    def advance_async(self):
        """advanceTimeSpan without waiting for the device (``wait`` completes it: timing, the NaN check)."""
        self.initialize()
        self._prepare_advance()
        self._call(N.lib().fdm_advance_async, self._start, self._end)

    def wait(self):
        self._call(N.lib().fdm_wait)

    def wait_for(self, timeout_s: float) -> bool:
        """``wait`` for at most ``timeout_s`` seconds: True once the advance is complete, False if it is still
        running (it stays enqueued; a later ``wait``/``wait_for`` completes it)."""
        rc = N.lib().fdm_wait_for(self._h, float(timeout_s))
        if rc == N.FDM_ERR_TIMEOUT:
            return False
        N.check(rc, self._h)
        return True

    def run(self):
        self.initialize()
        self.advanceTimeSpan()

    def reset(self):
        self.close()

    def saveFiberDataCheckpoint(self):
        self._call(N.lib().fdm_checkpoint_save)

    def restoreFiberDataCheckpoint(self):
        self._call(N.lib().fdm_checkpoint_restore)

    # -- data -------------------------------------------------------------------------------------
    def states(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """All states [state, node] (FP64); ``out`` reuses a C-contiguous float64 array of that shape."""
        ns = model_sizes(self.system.model)[0]
        if out is None or out.shape != (ns, self.system.n_nodes) or out.dtype != np.float64 \
                or not out.flags.c_contiguous:
            out = np.empty((ns, self.system.n_nodes))
        self._call(N.lib().fdm_get_states, N.ptr(out, C.c_double))
        return out

    def pinned_states(self) -> np.ndarray:
        """An array for all states [state, node] in page-locked host memory: ``set_states`` and
        ``states(out=...)`` move it by DMA without the staging copy (the values are the same either way)."""
        return N.pinned_array((model_sizes(self.system.model)[0], self.system.n_nodes))

    def set_states(self, states: np.ndarray):
        st = np.ascontiguousarray(states, np.float64)
        self._call(N.lib().fdm_set_states, N.ptr(st, C.c_double))

    def vm(self) -> np.ndarray:
        out = np.zeros(self.system.n_nodes)
        self._call(N.lib().fdm_get_vm, N.ptr(out, C.c_double))
        return out

    def algebraics(self) -> np.ndarray:
        k = len(self.system.algebraics_for_transfer)
        out = np.zeros((max(k, 1), self.system.n_nodes))
        if k:
            self._call(N.lib().fdm_get_algebraics, N.ptr(out, C.c_double))
        return out[:k]

    def parameters(self) -> np.ndarray:
        npar = model_sizes(self.system.model)[2]
        out = np.zeros((max(npar, 1), self.system.n_nodes))
        if npar:
            self._call(N.lib().fdm_get_parameters, N.ptr(out, C.c_double))
        return out[:npar]

    def set_parameters(self, params: np.ndarray):
        p = np.ascontiguousarray(params, np.float64)
        self._call(N.lib().fdm_set_parameters, N.ptr(p, C.c_double))

    def set_prefactor(self, prefactor: np.ndarray):
        p = np.ascontiguousarray(prefactor, np.float64)
        self._call(N.lib().fdm_set_prefactor, N.ptr(p, C.c_double))

    def trace(self) -> np.ndarray:
        n = C.c_int64()
        self._call(N.lib().fdm_get_trace, None, C.byref(n))
        out = np.zeros((max(n.value, 1), max(len(self.trace_nodes), 1)))
        if n.value and len(self.trace_nodes):
            self._call(N.lib().fdm_get_trace, N.ptr(out, C.c_double), C.byref(n))
        return out[:n.value, :len(self.trace_nodes)]

    def set_trace(self, nodes, capacity: int):
        """Traces Vm at ``nodes`` after each Strang step from now on (``capacity`` steps; rows count from here)."""
        self.initialize()
        self.trace_nodes = np.ascontiguousarray(nodes, np.int64)
        self.trace_capacity = int(capacity)
        self._call(N.lib().fdm_set_trace, len(self.trace_nodes), N.ptr(self.trace_nodes, C.c_int64),
                   self.trace_capacity)

    def record_activation(self, threshold: float = 0.0, capacity: int = 16):
        """Records, on the traced nodes, the Strang steps (trace rows) after which Vm rose above ``threshold``
        (fdm_set_activation_recording); ``capacity`` rows per node are kept, all crossings are counted."""
        self.initialize()
        self._act_cap = int(capacity)
        self._call(N.lib().fdm_set_activation_recording, float(threshold), self._act_cap)

    def activation_steps(self):
        """(counts [traced node], steps [traced node, capacity]; -1 where none) of record_activation."""
        n = len(self.trace_nodes)
        counts = np.zeros(max(n, 1), np.int32)
        steps = np.zeros((max(n, 1), max(self._act_cap, 1)), np.int32)
        self._call(N.lib().fdm_get_activation_steps, N.ptr(counts, C.c_int), N.ptr(steps, C.c_int))
        return counts[:n], steps[:n, :self._act_cap]

    def rewind(self):
        """Back to the start time: time-stepping state and stimulation machine reset, states kept."""
        self._call(N.lib().fdm_rewind)

    # -- adjoint ----------------------------------------------------------------------------------
    def adjoint_forward(self, t_start: float, t_end: float, checkpoint_every: int, sensor_nodes) -> np.ndarray:
        """Checkpointed FP64 forward run; returns Vm at the sensor nodes after every Strang step."""
        self.initialize()
        sn = np.ascontiguousarray(sensor_nodes, np.int64)
        self._sensors = sn
        self._call(N.lib().fdm_adjoint_forward, float(t_start), float(t_end), int(checkpoint_every), len(sn),
                   N.ptr(sn, C.c_int64))
        n = C.c_int64()
        self._call(N.lib().fdm_get_trace, None, C.byref(n))
        out = np.zeros((max(n.value, 1), max(len(sn), 1)))
        if n.value and len(sn):
            self._call(N.lib().fdm_get_trace, N.ptr(out, C.c_double), C.byref(n))
        return out[:n.value, :len(sn)]

    def adjoint_backward(self, trace_grad: np.ndarray) -> Dict[str, np.ndarray]:
        """Gradients of a loss whose derivative w.r.t. the recorded trace is trace_grad [steps, sensors]."""
        s = self.system
        ns, na, npar = model_sizes(s.model)[:3]
        tg = np.ascontiguousarray(trace_grad, np.float64)
        gpf = np.zeros(s.n_fibers)
        gp = np.zeros((max(npar, 1), s.n_nodes))
        g0 = np.zeros((ns, s.n_nodes))
        self._call(N.lib().fdm_adjoint_backward, N.ptr(tg, C.c_double), N.ptr(gpf, C.c_double),
                   N.ptr(gp, C.c_double), N.ptr(g0, C.c_double))
        return {"prefactor": gpf, "parameters": gp[:npar], "states0": g0}

    def adjoint_release(self):
        """Free the adjoint's checkpoints and replay buffers (the solver keeps its state)."""
        self._call(N.lib().fdm_adjoint_release)

    def adjoint_timing_ms(self) -> float:
        v = C.c_double()
        self._call(N.lib().fdm_adjoint_timing, C.byref(v))
        return v.value

    def equilibrium_state(self):
        """(statuses of all point buffers, per-rank counts of inactive buffers) of the equilibrium skip
        (0 inactive, 1 neighbor_is_active, 2 active)."""
        n = C.c_int64()
        self._call(N.lib().fdm_get_equilibrium_state, C.byref(n), None, None)
        st = np.zeros(max(n.value, 1), np.uint8)
        cnt = np.zeros(max(self.system.n_ranks, 1), np.int32)
        self._call(N.lib().fdm_get_equilibrium_state, C.byref(n), N.ptr(st, C.c_uint8), N.ptr(cnt, C.c_int))
        return st[:n.value], cnt

    def clamp_nodes(self):
        nf = self.system.n_fibers
        first = np.zeros(nf, np.int64)
        cnt = np.zeros(nf, np.int32)
        ev = np.zeros(nf, np.uint8)
        self._call(N.lib().fdm_get_clamp_nodes, N.ptr(first, C.c_int64), N.ptr(cnt, C.c_int), N.ptr(ev, C.c_uint8))
        return first, cnt, ev

    def fused_layout(self) -> Dict[str, int]:
        """The fused kernel's launch: CTA size, nodes per thread, CTAs per fiber (> 1: cluster mode), CTAs."""
        t, m, c, b = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self._call(N.lib().fdm_fused_layout, C.byref(t), C.byref(m), C.byref(c), C.byref(b))
        return {"threads": t.value, "nodes_per_thread": m.value, "cluster_size": c.value, "n_blocks": b.value}

    def split_steps(self) -> int:
        return int(N.lib().fdm_split_steps(self._h))

    def timing(self) -> Dict[str, float]:
        a, b, c, d = C.c_double(), C.c_int64(), C.c_double(), C.c_int64()
        self._call(N.lib().fdm_get_timing, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return {"main_kernel_ms": a.value, "main_kernel_launches": b.value, "advance_ms": c.value,
                "kernel_launches": d.value}

    def reset_timing(self):
        self._call(N.lib().fdm_reset_timing)

    def compute_state_information(self) -> np.ndarray:
        """"computeStateInformation" per node (communication.tpp:277-290): the status of the node's point
        buffer (0 inactive, 1 neighbor_is_active, 2 active), -1 on fibers not stimulated yet under
        onlyComputeIfHasBeenStimulated."""
        out = np.empty(self.system.n_nodes, np.float64)
        self._call(N.lib().fdm_get_compute_state_information, N.ptr(out, C.c_double))
        return out

    def data(self) -> Dict[str, np.ndarray]:
        """The fiber data the reference transfers out (statesForTransfer / algebraicsForTransfer, and
        computeStateInformation when the diffusion solver has the extra slot)."""
        st = self.states()
        d = {"Vm": st[0], "states": st[list(self.system.states_for_transfer)], "algebraics": self.algebraics()}
        if self.system.compute_state_information:
            d["computeStateInformation"] = self.compute_state_information()
        return d
