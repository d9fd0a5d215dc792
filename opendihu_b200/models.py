"""Run-time model modules: CellML models and parameter variants that are not built into libfdm_b200.so.

The reference generates C++ code from the CellML model file and the settings' parameter choice
(parametersUsedAsAlgebraic / parametersUsedAsConstant), compiles it and loads the library at run time
(fast_monodomain_solver_gpu.tpp:106-205; 00_source_code_generator_base.cpp:45-176).  This module does the same
for the device code: it emits the model's device functions for the requested variant (cellml.emit_cuda_model),
instantiates the library's kernel templates for them in a translation unit of its own
(csrc/fdm_model_module.cuh), compiles that with nvcc for sm_100a into a shared library and registers it with
the running library (fdm_register_model_library).  Modules are cached by the hash of their source and of the
library headers they are compiled against, in $FDM_MODEL_CACHE or _build/models/ of the repository.

The built-in models carry their parsed equations in their generated description
(csrc/generated/<model>_<variant>.json), so every parameter variant of them can be generated without the model
file; other models need their OpenCOR C file.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
import threading
from typing import Dict, Optional, Sequence, Tuple

from . import _native as N
from . import build as B
from . import cellml as CM

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
_LOCK = threading.Lock()
#: registered module name -> (model id, parametersUsedAsAlgebraic, parametersUsedAsConstant, parsed model)
_MODULES: Dict[str, Tuple[int, tuple, tuple, "CM.Model"]] = {}

# library headers a module is compiled against (part of its cache key; the ABI check at load time covers the rest)
_HEADERS = ("fdm_kernels.cuh", "fdm_equilibrium.cuh", "fdm_internal.h", "fdm_math.cuh", "fdm_model_launch.cuh",
            "fdm_model_module.cuh")


def cache_dir() -> str:
    return os.environ.get("FDM_MODEL_CACHE") or os.path.join(B.ROOT, "_build", "models")


def builtin_variant(model_name: str, params_alg: Sequence[int], params_const: Sequence[int]) -> bool:
    """True if the library carries this model with a variant whose parameter slots cover the request: the same
    algebraic parameters and constant parameters among its own (those not requested keep their defaults)."""
    from .solver import VARIANT_PARAMETERS
    if model_name not in VARIANT_PARAMETERS:
        return False
    pa_var, pc_var = VARIANT_PARAMETERS[model_name]
    return tuple(params_alg) == tuple(pa_var) and all(c in pc_var for c in params_const)


def module_name(model: "CM.Model", params_alg: Sequence[int], params_const: Sequence[int]) -> str:
    return f"{CM._ident(model)}_{CM.variant_tag(params_alg, params_const)}"


def load_model(model_name: str, params_alg: Sequence[int] = (), params_const: Sequence[int] = (),
               model_file: Optional[str] = None, verbose: bool = False) -> str:
    """Make the model variant available to the library and return the name to use as FiberSystem.model.

    A built-in model with a variant the library carries is returned as it is.  Any other variant of a built-in
    model, or a model given by its OpenCOR C file, is generated, compiled (once; cached) and registered."""
    params_alg, params_const = tuple(int(x) for x in params_alg), tuple(int(x) for x in params_const)
    if model_file is None and builtin_variant(model_name, params_alg, params_const):
        return model_name
    if model_file is not None and os.path.exists(model_file):
        model = CM.parse_model_file(model_file)
    else:
        try:
            model = CM.builtin_model(model_name)
        except KeyError:
            raise ValueError(f"model {model_name!r}: not built into the library and its model file "
                             f"{model_file!r} does not exist") from None
    for a in params_alg:
        if not 0 <= a < model.n_algebraics:
            raise ValueError(f"model {model.name}: parametersUsedAsAlgebraic index {a} out of range")
    for c in params_const:
        if not 0 <= c < model.n_constants:
            raise ValueError(f"model {model.name}: parametersUsedAsConstant index {c} out of range")
    name = module_name(model, params_alg, params_const)
    with _LOCK:
        if name in _MODULES:
            return name
        path = _build_module(model, params_alg, params_const, name, verbose)
        mid = ctypes.c_int()
        N.check(N.lib().fdm_register_model_library(path.encode(), ctypes.byref(mid)))
        _MODULES[name] = (mid.value, params_alg, params_const, model)
        N.MODEL_IDS[name] = mid.value
    return name


def module_info(name: str):
    """(model id, parametersUsedAsAlgebraic, parametersUsedAsConstant, parsed model) of a loaded module."""
    return _MODULES[name]


def _source(model, params_alg, params_const, name) -> Tuple[str, str]:
    header = CM.emit_cuda_model(model, params_alg, params_const)
    # the registered name identifies the variant (the built-in models keep their plain names)
    header = header.replace(f'static constexpr const char* name = "{model.name}";',
                            f'static constexpr const char* name = "{name}";', 1)
    struct = f"fdm_model_{CM._ident(model)}_{CM.variant_tag(params_alg, params_const)}"
    unit = ("// Run-time model module generated by opendihu_b200/models.py; do not edit.\n"
            '#include "model.cuh"\n'
            f"#define FDM_MODULE_MODEL {struct}\n"
            '#include "fdm_model_module.cuh"\n')
    return header, unit


def _build_module(model, params_alg, params_const, name, verbose) -> str:
    header, unit = _source(model, params_alg, params_const, name)
    h = hashlib.sha1()
    for text in (header, unit, " ".join(B.NVCC_FLAGS)):
        h.update(text.encode())
    for f in _HEADERS:
        with open(os.path.join(CSRC, f), "rb") as fh:
            h.update(fh.read())
    d = os.path.join(cache_dir(), f"{name}-{h.hexdigest()[:16]}")
    lib = os.path.join(d, "module.so")
    if os.path.exists(lib):
        return lib
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "model.cuh"), "w") as f:
        f.write(header)
    with open(os.path.join(d, "module.cu"), "w") as f:
        f.write(unit)
    tmp = lib + f".tmp{os.getpid()}"
    cmd = [B.nvcc()] + B.NVCC_FLAGS + ["-I", CSRC, "-I", os.path.join(CSRC, "generated"), "-I", d,
                                        "-shared", "-o", tmp, os.path.join(d, "module.cu")]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for the model module {name}:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    return lib
