"""Input-file parsers restated from fast_monodomain_solver_initialization.tpp:145-234."""
import json
import os

import numpy as np
import pytest

from opendihu_b200 import inputs

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cellml_golden.json")))


def test_firing_times_last_line_needs_newline():
    assert inputs.parse_firing_times("1 0 1\n0 1 0") == [[1, 0, 1]]
    assert inputs.parse_firing_times("1 0 1\n0 1 0\n") == [[1, 0, 1], [0, 1, 0]]


def test_firing_times_separators_and_trailing_space():
    assert inputs.parse_firing_times("1\t0  1 \n") == [[1, 0, 1]]
    assert inputs.parse_firing_times("0 2 x1\n") == [[0, 1, 1]]


def test_fiber_distribution_newline_is_not_a_separator():
    assert inputs.parse_fiber_distribution("1 2\n3 4") == [1, 2, 4]
    assert inputs.parse_fiber_distribution("7") == [7]
    assert inputs.parse_fiber_distribution("8 4 8 ") == [8, 4, 8]
    assert inputs.parse_fiber_distribution("8 4 \n") == [8, 4, 0]


def test_ragged_rows_to_matrix_keeps_row_modulo():
    rows = [[1, 0], [0, 1, 1]]
    m = inputs.firing_matrix(rows)
    assert m.shape == (2, 6)
    for mu in range(20):
        for r, row in enumerate(rows):
            assert m[r, mu % m.shape[1]] == row[mu % len(row)]


def test_reference_input_summaries_roundtrip(tmp_path):
    # writer + parser reproduce the shapes the reference's own fixtures have
    g = GOLD["MU_firing_times_always.txt"]
    p = tmp_path / "ft.txt"
    inputs.write_firing_times(str(p), np.ones((g["rows"], g["cols"][0]), np.uint8))
    rows = inputs.parse_firing_times(p.read_text())
    assert len(rows) == g["rows"] and [len(r) for r in rows] == g["cols"] and sum(map(sum, rows)) == g["sum"]
    g = GOLD["MU_fibre_distribution_10MUs.txt"]
    p = tmp_path / "fd.txt"
    mus = list(g["first"]) + [1] * (g["n"] - 20) + list(g["last"])
    inputs.write_fiber_distribution(str(p), mus)
    back = inputs.parse_fiber_distribution(p.read_text())
    assert len(back) == g["n"] and back[:10] == g["first"] and back[-10:] == g["last"]


def test_synthetic_generators_are_seeded():
    a = inputs.exponential_mu_distribution(4096, 100, seed=0)
    b = inputs.exponential_mu_distribution(4096, 100, seed=0)
    assert (a == b).all() and a.min() >= 1 and a.max() <= 100
    f = inputs.poisson_firing_times(100, 100.0, 0.1, 10, 40, seed=0)
    assert f.shape == (11, 101) and set(np.unique(f)) <= {0, 1}
