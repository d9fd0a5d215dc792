"""Run-time model modules (no GPU needed): a parameter variant the library does not carry is generated from
the model's equations, compiled with nvcc for sm_100a into a module library and registered with the running
library, as the reference generates, compiles and loads its model library at run time
(fast_monodomain_solver_gpu.tpp:106-205).  The settings layer does this for any parametersUsedAsAlgebraic /
parametersUsedAsConstant choice."""
import numpy as np
import pytest

import helpers as H
from opendihu_b200 import _native as N
from opendihu_b200 import cellml as CM
from opendihu_b200 import models as MD
from opendihu_b200 import solver as S
from test_only_if_stimulated import reference_settings


def test_builtin_variants_need_no_module():
    assert MD.load_model(H.HH, (), (2, 3, 4)) == H.HH
    assert MD.load_model(H.HH, (), (3, 4)) == H.HH          # covered by the built-in variant's slots
    assert MD.load_model(H.SHORTEN, (32,), (65,)) == H.SHORTEN


def test_variant_module_is_built_and_registered():
    name = MD.load_model(H.HH, (), (3, 5))                  # g_Na and g_L as parameters, g_K and i_Stim constant
    assert name == "hodgkin_huxley_1952_anone_c3_5"
    mid = N.MODEL_IDS[name]
    assert mid >= 2                                         # after the built-in models
    ns, na, npar, init, defaults = N.model_info(mid)
    assert (ns, na, npar) == (4, 9, 2)
    np.testing.assert_array_equal(init, [-75, 0.05, 0.6, 0.325])
    np.testing.assert_array_equal(defaults, [120.0, 0.3])
    assert MD.load_model(H.HH, (), (3, 5)) == name          # loaded once
    assert N.MODEL_IDS[name] == mid


def test_builtin_model_equations_survive_the_round_trip():
    m = CM.builtin_model(H.HH)
    assert (m.n_states, m.n_algebraics, m.n_constants) == (4, 9, 9)
    j = CM.model_to_json(m)
    m2 = CM.model_from_json(j)
    assert CM.emit_cuda_model(m2, (), (3, 5)) == CM.emit_cuda_model(m, (), (3, 5))
    assert m2.constants == m.constants


def test_settings_with_a_variant_the_library_does_not_carry():
    cfg = reference_settings(n_fibers=2, onlyComputeIfHasBeenStimulated=False,
                             disableComputationWhenStatesAreCloseToEquilibrium=False)
    for inst in cfg["RepeatedCall"]["MultipleInstances"]["instances"][0]["StrangSplitting"]["Term1"][
            "MultipleInstances"]["instances"]:
        inst["Heun"]["CellML"]["parametersUsedAsConstant"] = [3, 5]
        inst["Heun"]["CellML"]["parametersInitialValues"] = [110.0, 0.25]
    s = S.parse_settings(cfg)
    assert s.model == "hodgkin_huxley_1952_anone_c3_5"
    assert s.parameters.shape == (2, s.n_nodes)
    np.testing.assert_array_equal(s.parameters[:, 0], [110.0, 0.25])


def test_out_of_range_parameter_is_refused():
    with pytest.raises(ValueError):
        MD.load_model(H.HH, (), (9,))
