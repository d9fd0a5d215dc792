"""ctypes binding of libfdm_b200.so (the C ABI declared in include/fdm_b200.h).

There is no CPU fallback: if the library is missing or has no CUDA device, the solver raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libfdm_b200.so")

FDM_OK = 0
FDM_ERR_ARG = 1
FDM_ERR_CUDA = 2
FDM_ERR_NAN = 3
FDM_ERR_UNSUPPORTED = 4
FDM_ERR_NO_DEVICE = 5
FDM_ERR_TIMEOUT = 6

MODEL_IDS = {"hodgkin_huxley_1952": 0, "shorten_ocallaghan_davidson_soboleva_2007": 1}

#: every symbol include/fdm_b200.h declares
EXPORTED = [
    "fdm_config_default", "fdm_create", "fdm_destroy", "fdm_last_error", "fdm_model_info",
    "fdm_model_parameter_defaults", "fdm_set_fibers", "fdm_set_prefactor", "fdm_set_parameters",
    "fdm_get_parameters", "fdm_set_states", "fdm_get_states", "fdm_get_vm", "fdm_set_stimulation",
    "fdm_get_clamp_nodes", "fdm_set_algebraics_for_transfer", "fdm_get_algebraics", "fdm_set_trace",
    "fdm_get_trace", "fdm_advance", "fdm_split_steps", "fdm_get_timing", "fdm_reset_timing",
    "fdm_checkpoint_save", "fdm_checkpoint_restore", "fdm_fused_shapes", "fdm_diffusion_solve",
    "fdm_diffusion_solve_noalloc", "fdm_compat_configure", "fdm_compat_release", "fdm_adjoint_forward",
    "fdm_adjoint_backward", "fdm_adjoint_release", "fdm_adjoint_timing", "fdm_rewind", "fdm_set_clamp_nodes",
    "fdm_select_clamp_nodes", "fdm_select_gate_codes", "fdm_set_gate_codes", "fdm_get_equilibrium_state",
    "fdm_cellml_rhs_device", "fdm_cellml_rhs_configure", "fdm_fused_cluster_shapes", "fdm_fused_layout",
    "fdm_get_compute_state_information", "fdm_advance_async", "fdm_wait", "fdm_wait_for", "fdm_repeated_call_plan",
    "fdm_advance_pieces", "fdm_set_stimulation_log", "fdm_get_stimulation_log",
    "fdm_model_equilibrium", "fdm_emg_set_preconditioner", "fdm_emg_create", "fdm_emg_destroy", "fdm_emg_last_error",
    "fdm_emg_potential_flow", "fdm_emg_set_direction", "fdm_emg_set_conductivity", "fdm_emg_set_fiber_mapping",
    "fdm_emg_map_fibers", "fdm_emg_map_values", "fdm_emg_set_vm", "fdm_emg_solve", "fdm_emg_get",
    "fdm_emg_get_stencil", "fdm_emg_timing", "fdm_debug_fail_allocation", "fdm_set_activation_recording",
    "fdm_get_activation_steps", "fdm_register_model_library", "fdm_host_alloc", "fdm_host_free",
]

#: fdm_emg_get fields of include/fdm_b200.h
EMG_PHI_E, EMG_VM, EMG_RHS, EMG_FLOW_POTENTIAL, EMG_DIRECTION = 0, 1, 2, 3, 4
EMG_PRECOND_JACOBI, EMG_PRECOND_MULTIGRID = 0, 1

#: FDM_NOALLOC_MAX_NODES of include/fdm_b200.h
NOALLOC_MAX_NODES = 262144


class FdmError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[fdm error {code}] {message}")
        self.code = code


class Config(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("diffusion_scheme", C.c_int), ("method", C.c_int),
        ("reaction_precision", C.c_int), ("approximate_exponential_function", C.c_int),
        ("clamp_rule", C.c_int), ("vc_width", C.c_int), ("n_ranks", C.c_int),
        ("stimulus_mode", C.c_int), ("stimulus_parameter", C.c_int), ("stimulus_value", C.c_double),
        ("value_for_stimulated_point", C.c_double), ("dt_repeated_call", C.c_double),
        ("dt_splitting", C.c_double), ("dt_0d", C.c_double), ("dt_1d", C.c_double),
        ("steps_per_launch", C.c_int), ("threads_per_block", C.c_int), ("nodes_per_thread", C.c_int),
        ("check_nan", C.c_int), ("profile", C.c_int), ("device", C.c_int), ("use_graph", C.c_int),
        ("only_compute_if_stimulated", C.c_int), ("skip_close_to_equilibrium", C.c_int),
        ("cluster_size", C.c_int),
    ]


_lib = None


def lib() -> C.CDLL:
    """Load the library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FdmError(FDM_ERR_ARG, f"{LIB_PATH} is missing; build it with opendihu_b200.build.build()")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    d = C.POINTER(C.c_double)
    i64 = C.POINTER(C.c_int64)
    i32 = C.POINTER(C.c_int)
    u8 = C.POINTER(C.c_uint8)
    sig = {
        "fdm_config_default": (None, [C.POINTER(Config)]),
        "fdm_create": (C.c_int, [C.POINTER(Config), C.POINTER(P)]),
        "fdm_destroy": (C.c_int, [P]),
        "fdm_last_error": (C.c_char_p, [P]),
        "fdm_model_info": (C.c_int, [C.c_int, i32, i32, i32, d]),
        "fdm_model_parameter_defaults": (C.c_int, [C.c_int, d]),
        "fdm_set_fibers": (C.c_int, [P, C.c_int, i64, d, d]),
        "fdm_set_prefactor": (C.c_int, [P, d]),
        "fdm_set_parameters": (C.c_int, [P, d]),
        "fdm_get_parameters": (C.c_int, [P, d]),
        "fdm_set_states": (C.c_int, [P, d]),
        "fdm_get_states": (C.c_int, [P, d]),
        "fdm_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(C.c_void_p)]),
        "fdm_host_free": (C.c_int, [C.c_void_p]),
        "fdm_get_vm": (C.c_int, [P, d]),
        "fdm_set_stimulation": (C.c_int, [P, u8, C.c_int, C.c_int, i32, i32, d, d, d, d, C.c_int]),
        "fdm_get_clamp_nodes": (C.c_int, [P, i64, i32, u8]),
        "fdm_set_algebraics_for_transfer": (C.c_int, [P, C.c_int, i32]),
        "fdm_get_algebraics": (C.c_int, [P, d]),
        "fdm_set_trace": (C.c_int, [P, C.c_int, i64, C.c_int64]),
        "fdm_get_trace": (C.c_int, [P, d, i64]),
        "fdm_set_activation_recording": (C.c_int, [P, C.c_double, C.c_int]),
        "fdm_register_model_library": (C.c_int, [C.c_char_p, i32]),
        "fdm_get_activation_steps": (C.c_int, [P, i32, i32]),
        "fdm_advance": (C.c_int, [P, C.c_double, C.c_double]),
        "fdm_advance_async": (C.c_int, [P, C.c_double, C.c_double]),
        "fdm_wait": (C.c_int, [P]),
        "fdm_wait_for": (C.c_int, [P, C.c_double]),
        "fdm_debug_fail_allocation": (C.c_int, [C.c_int64]),
        "fdm_repeated_call_plan": (C.c_int, [P, C.c_double, C.c_double, C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
        "fdm_advance_pieces": (C.c_int, [P, C.c_double, C.c_double, C.c_int64, C.c_int64]),
        "fdm_set_stimulation_log": (C.c_int, [P, C.c_int64]),
        "fdm_model_equilibrium": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_double,
                                            C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]),
        "fdm_get_stimulation_log": (C.c_int, [P, C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_int)]),
        "fdm_split_steps": (C.c_int64, [P]),
        "fdm_get_timing": (C.c_int, [P, d, i64, d, i64]),
        "fdm_reset_timing": (C.c_int, [P]),
        "fdm_checkpoint_save": (C.c_int, [P]),
        "fdm_checkpoint_restore": (C.c_int, [P]),
        "fdm_fused_shapes": (C.c_int, [i32, i32, C.c_int]),
        "fdm_fused_cluster_shapes": (C.c_int, [i32, i32, C.c_int]),
        "fdm_fused_layout": (C.c_int, [P, i32, i32, i32, i32]),
        "fdm_get_compute_state_information": (C.c_int, [P, d]),
        "fdm_emg_create": (C.c_int, [C.c_int, C.c_int, C.c_int, d, C.c_int, C.POINTER(P)]),
        "fdm_emg_destroy": (C.c_int, [P]),
        "fdm_emg_last_error": (C.c_char_p, [P]),
        "fdm_emg_potential_flow": (C.c_int, [P, C.c_int64, i64, d, C.c_int, C.c_double, C.c_double, C.c_int, i32]),
        "fdm_emg_set_direction": (C.c_int, [P, d]),
        "fdm_emg_set_conductivity": (C.c_int, [P, C.c_int64, d, C.c_int64, d, C.c_int]),
        "fdm_emg_set_fiber_mapping": (C.c_int, [P, C.c_int64, d, C.c_double, C.c_double, i64]),
        "fdm_emg_map_fibers": (C.c_int, [P, P]),
        "fdm_emg_map_values": (C.c_int, [P, d]),
        "fdm_emg_set_vm": (C.c_int, [P, d]),
        "fdm_emg_solve": (C.c_int, [P, C.c_double, C.c_double, C.c_int, C.c_int, i32, d]),
        "fdm_emg_get": (C.c_int, [P, C.c_int, d]),
        "fdm_emg_get_stencil": (C.c_int, [P, C.c_int, d]),
        "fdm_emg_timing": (C.c_int, [P, d, i32, d]),
        "fdm_emg_set_preconditioner": (C.c_int, [P, C.c_int, i32]),
        "fdm_diffusion_solve": (C.c_int, [C.c_int, C.c_int64, P, P, P, C.c_double, C.c_int, P, P]),
        "fdm_diffusion_solve_noalloc": (C.c_int, [C.c_int, C.c_int64, P, P, P, C.c_double, C.c_int, P, P]),
        "fdm_compat_configure": (C.c_int, [C.c_int] * 13),
        "fdm_adjoint_forward": (C.c_int, [P, C.c_double, C.c_double, C.c_int, C.c_int, i64]),
        "fdm_adjoint_backward": (C.c_int, [P, d, d, d, d]),
        "fdm_adjoint_release": (C.c_int, [P]),
        "fdm_adjoint_timing": (C.c_int, [P, d]),
        "fdm_rewind": (C.c_int, [P]),
        "fdm_set_clamp_nodes": (C.c_int, [P, i64, i32, u8]),
        "fdm_select_clamp_nodes": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, i64, i32, i64, i32, u8]),
        "fdm_select_gate_codes": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, i64, i32, i32]),
        "fdm_set_gate_codes": (C.c_int, [P, i32]),
        "fdm_get_equilibrium_state": (C.c_int, [P, i64, u8, i32]),
        "fdm_cellml_rhs_device": (C.c_int, [C.c_int, C.c_int, C.c_int64, C.c_double, P, P, P, P, P]),
        "fdm_cellml_rhs_configure": (C.c_int, [C.c_int, C.c_int64, C.c_int, C.c_int]),
        "computeCellMLRightHandSide": (None, [P, C.c_double, d, d, d, d]),
        "fdm_compat_release": (C.c_int, []),
        "initializeArrays": (None, [d, i32, i32, C.c_char_p, d, i32, i32, d, d, d, d]),
        "computeMonodomain": (None, [C.POINTER(C.c_float), d, d, C.POINTER(C.c_float), C.c_double, C.c_double,
                                     C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def check(rc: int, handle=None):
    if rc != FDM_OK:
        msg = lib().fdm_last_error(handle)
        raise FdmError(rc, msg.decode() if msg else "")


class _PinnedBuffer:
    """Page-locked host memory from fdm_host_alloc, exposed to numpy and released with the last array over it."""

    def __init__(self, shape, dtype):
        self.ptr = None
        dt = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dt.itemsize
        p = C.c_void_p()
        check(lib().fdm_host_alloc(max(nbytes, 1), C.byref(p)))
        self.ptr = p.value
        self.__array_interface__ = {"shape": tuple(int(n) for n in shape), "typestr": dt.str,
                                    "data": (self.ptr, False), "version": 3}

    def __del__(self):
        if self.ptr:
            try:
                lib().fdm_host_free(C.c_void_p(self.ptr))
            except Exception:  # noqa: BLE001 - interpreter shutdown: the library may be gone already
                pass
            self.ptr = None


def pinned_array(shape, dtype=np.float64) -> np.ndarray:
    """A C-contiguous array in page-locked host memory (fdm_host_alloc): the state transfers DMA it directly."""
    return np.asarray(_PinnedBuffer(shape, dtype))


def default_config() -> Config:
    c = Config()
    lib().fdm_config_default(C.byref(c))
    return c


def model_info(model: int):
    ns, na, npar = C.c_int(), C.c_int(), C.c_int()
    init = np.zeros(128)
    check(lib().fdm_model_info(model, C.byref(ns), C.byref(na), C.byref(npar), ptr(init, C.c_double)))
    defaults = np.zeros(max(npar.value, 1))
    check(lib().fdm_model_parameter_defaults(model, ptr(defaults, C.c_double)))
    return ns.value, na.value, npar.value, init[:ns.value].copy(), defaults[:npar.value].copy()


def fused_shapes(cluster: bool = False):
    """(threads, nodes per thread) of the built fused-kernel shapes (``cluster``: of its cluster mode)."""
    t = np.zeros(64, np.int32)
    m = np.zeros(64, np.int32)
    fn = lib().fdm_fused_cluster_shapes if cluster else lib().fdm_fused_shapes
    n = fn(ptr(t, C.c_int), ptr(m, C.c_int), 64)
    return [(int(t[i]), int(m[i])) for i in range(n)]


def select_clamp_nodes(rule: int, vc_width: int, n_ranks: int, fiber_offsets, stimulation_point_index):
    """Host-only junction clamp selection of the library (first node, count, machine evaluated per fiber)."""
    off = np.ascontiguousarray(fiber_offsets, np.int64)
    c = np.ascontiguousarray(stimulation_point_index, np.int32)
    nf = len(off) - 1
    first = np.zeros(max(nf, 1), np.int64)
    cnt = np.zeros(max(nf, 1), np.int32)
    ev = np.zeros(max(nf, 1), np.uint8)
    check(lib().fdm_select_clamp_nodes(rule, vc_width, n_ranks, nf, ptr(off, C.c_int64), ptr(c, C.c_int),
                                       ptr(first, C.c_int64), ptr(cnt, C.c_int), ptr(ev, C.c_uint8)))
    return first[:nf], cnt[:nf], ev[:nf]


def select_gate_codes(rule: int, vc_width: int, n_ranks: int, fiber_offsets, stimulation_point_index):
    """Host-only per-node codes (attributed fiber * 4 + class) of onlyComputeIfHasBeenStimulated."""
    off = np.ascontiguousarray(fiber_offsets, np.int64)
    c = np.ascontiguousarray(stimulation_point_index, np.int32)
    n = int(off[-1]) if len(off) else 0
    codes = np.zeros(max(n, 1), np.int32)
    check(lib().fdm_select_gate_codes(rule, vc_width, n_ranks, len(off) - 1, ptr(off, C.c_int64), ptr(c, C.c_int),
                                      ptr(codes, C.c_int)))
    return codes[:n]
