"""The C ABI library loads and exports every symbol include/fdm_b200.h declares (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import helpers as H
from opendihu_b200 import _native as N

HEADER = os.path.join(H.ROOT, "include", "fdm_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fdm_[a-z0-9_]+)\s*\(", text)) | set(
        re.findall(r"\b(initializeArrays|computeMonodomain|computeCellMLRightHandSide)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = N.lib()
    missing = [f for f in declared_functions() if not hasattr(L, f)]
    assert not missing, missing


def test_binding_list_matches_header():
    assert sorted(N.EXPORTED) == [f for f in declared_functions() if f.startswith("fdm_")]


def test_model_info_without_device():
    ns, na, npar, init, defaults = N.model_info(N.MODEL_IDS[H.HH])
    assert (ns, na, npar) == (4, 9, 3)
    np.testing.assert_array_equal(init, [-75, 0.05, 0.6, 0.325])
    np.testing.assert_array_equal(defaults, [0.0, 120.0, 36.0])
    ns, na, npar, init, defaults = N.model_info(N.MODEL_IDS[H.SHORTEN])
    assert (ns, na, npar) == (56, 71, 2)


def test_create_fails_loudly_without_device_or_with_bad_config():
    cfg = N.default_config()
    cfg.model = 99
    h = C.c_void_p()
    rc = N.lib().fdm_create(C.byref(cfg), C.byref(h))
    assert rc == N.FDM_ERR_ARG and b"unknown model" in N.lib().fdm_last_error(None)
    cfg = N.default_config()
    cfg.model = N.MODEL_IDS[H.SHORTEN]
    cfg.method = 1
    assert N.lib().fdm_create(C.byref(cfg), C.byref(h)) == N.FDM_ERR_UNSUPPORTED


def test_fused_shapes_listed():
    shapes = N.fused_shapes()
    assert len(shapes) >= 4 and all(t % 32 == 0 and m >= 1 for t, m in shapes)
    cl = N.fused_shapes(cluster=True)
    assert len(cl) >= 1 and all(t % 32 == 0 and m >= 1 for t, m in cl)


@pytest.mark.parametrize("field,value,code", [
    ("cluster_size", 9, N.FDM_ERR_ARG), ("cluster_size", -1, N.FDM_ERR_ARG),
    ("method", 0, N.FDM_ERR_UNSUPPORTED),                             # cluster mode is a fused-kernel mode
    ("approximate_exponential_function", 1, N.FDM_ERR_UNSUPPORTED),
    ("only_compute_if_stimulated", 1, N.FDM_ERR_UNSUPPORTED)])
def test_cluster_mode_config_checked_before_the_device(field, value, code):
    cfg = N.default_config()
    cfg.method = 1
    cfg.cluster_size = 4
    setattr(cfg, field, value)
    h = C.c_void_p()
    assert N.lib().fdm_create(C.byref(cfg), C.byref(h)) == code
    assert b"cluster" in N.lib().fdm_last_error(None)


def test_host_alloc_fails_loudly_without_device_and_free_checks_its_pointer():
    import torch
    if torch.cuda.is_available():
        pytest.skip("the device form is tested in test_gpu_edge_cases.py")
    p = C.c_void_p()
    assert N.lib().fdm_host_alloc(1024, C.byref(p)) == N.FDM_ERR_NO_DEVICE
    assert p.value is None
    assert b"no CUDA device" in N.lib().fdm_last_error(None)
    assert N.lib().fdm_host_alloc(0, C.byref(p)) == N.FDM_ERR_ARG
    buf = np.zeros(4)
    assert N.lib().fdm_host_free(buf.ctypes.data_as(C.c_void_p)) == N.FDM_ERR_ARG
    assert N.lib().fdm_host_free(None) == N.FDM_OK
    with pytest.raises(N.FdmError):
        N.pinned_array((2, 3))
