"""The oracle's model right-hand sides against the reference's golden vectors.

The fixture tests/golden/cellml_golden.json holds the states the reference's own tests expect after
90001 explicit Euler steps (CellMLTest.HodgkinHuxleySimd / .ShortenOpenCOR in
testing/unit_testing/src/1_rank/cellml.cpp), compared there at an absolute 1e-13.
"""
import json
import os

import numpy as np

import helpers as H
from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cellml_golden.json")))


def test_hodgkin_huxley_explicit_euler_golden():
    g = GOLD["hodgkin_huxley_1952"]
    ee = GOLD["explicit_euler"]
    params = [g["parameters"]["I_Stim (CONSTANTS[2])"], 120.0, 36.0]
    s = O.explicit_euler_cell(H.HH, g["states_initial"], params, ee["dt"], ee["n_steps"])
    np.testing.assert_allclose(s, g["states_final"], rtol=0, atol=ee["tolerance"])


def test_shorten_explicit_euler_golden():
    g = GOLD["shorten_ocallaghan_davidson_soboleva_2007"]
    ee = GOLD["explicit_euler"]
    init = O.model_info(H.SHORTEN)[3]
    s = O.explicit_euler_cell(H.SHORTEN, init, [1000.0, 1.0], ee["dt"], ee["n_steps"])
    np.testing.assert_allclose(s, g["states_final"], rtol=0, atol=ee["tolerance"] * 1000)
    # relative agreement to a few ulps (the largest state is ~1.7e4)
    np.testing.assert_allclose(s, g["states_final"], rtol=1e-14, atol=1e-15)


def test_golden_vector_sizes():
    assert len(GOLD["hodgkin_huxley_1952"]["states_final"]) == 4
    assert len(GOLD["shorten_ocallaghan_davidson_soboleva_2007"]["states_final"]) == 56
