"""Input files of the FastMonodomainSolver: parsers and writers in the reference's formats.

Parsers restate FastMonodomainSolverBase::initializeFiringTimes
(core/src/specialized_solver/fast_monodomain_solver/fast_monodomain_solver_initialization.tpp:145-234),
including its corner cases:

* firing times file: one row per line, a line is only taken when it ends in a newline (a last line
  without one is ignored); entries are separated by a space or a tab, and after a separator every
  following non-digit character is skipped; each entry is ``atoi`` of the rest of the line.
* fiber distribution file: ``atoi`` of the text, then the text after the next space or tab, until
  there is none (a newline is *not* a separator).

Writers produce the same formats as the reference's generators (scripts/generate_firing_times.py,
scripts/generate_fiber_distribution.py): one line of space separated MU numbers, and rows of
space separated 0/1 flags.
"""
from __future__ import annotations

import math
from typing import List, Sequence

import numpy as np


def _atoi(s: str) -> int:
    i = 0
    n = len(s)
    while i < n and s[i] in " \t\n\r\v\f":
        i += 1
    sign = 1
    if i < n and s[i] in "+-":
        sign = -1 if s[i] == "-" else 1
        i += 1
    j = i
    while j < n and s[j].isdigit():
        j += 1
    return sign * int(s[i:j]) if j > i else 0


def parse_firing_times(text: str) -> List[List[int]]:
    rows: List[List[int]] = []
    while text:
        pos = text.find("\n")
        if pos < 0:
            break
        line = text[:pos]
        text = text[pos + 1:]
        row: List[int] = []
        while line:
            row.append(1 if _atoi(line) else 0)
            seps = [p for p in (line.find("\t"), line.find(" ")) if p >= 0]
            if not seps:
                break
            line = line[min(seps) + 1:]
            while line and not line[0].isdigit():
                line = line[1:]
        rows.append(row)
    if not rows:
        raise ValueError("Could not parse firing times.")
    return rows


def parse_fiber_distribution(text: str) -> List[int]:
    mus: List[int] = []
    while text:
        mus.append(_atoi(text))
        seps = [p for p in (text.find("\t"), text.find(" ")) if p >= 0]
        if not seps:
            break
        text = text[min(seps) + 1:]
    if not mus:
        raise ValueError("Could not parse motor units.")
    return mus


def firing_matrix(rows: List[List[int]], max_cols: int = 1 << 16) -> np.ndarray:
    """Rectangular uint8 matrix equivalent to the ragged rows.

    The reference indexes a row as ``row[mu % len(row)]`` (fast_monodomain_solver_compute.tpp:586); a
    matrix whose width is the least common multiple of the row lengths, each row repeated
    periodically, gives the same entry for every motor unit with one uniform ``mu % cols``.
    """
    lengths = [len(r) for r in rows]
    if min(lengths) == 0:
        raise ValueError("firing times file has an empty row")
    cols = 1
    for L in lengths:
        cols = cols * L // math.gcd(cols, L)
        if cols > max_cols:
            raise ValueError("firing times rows have incompatible lengths")
    out = np.zeros((len(rows), cols), np.uint8)
    for i, r in enumerate(rows):
        arr = np.asarray(r, np.uint8)
        out[i] = np.tile(arr, cols // len(r))
    return out


def write_fiber_distribution(path: str, mus: Sequence[int]) -> None:
    with open(path, "w") as f:
        f.write(" ".join(str(int(m)) for m in mus))


def write_firing_times(path: str, matrix: np.ndarray) -> None:
    with open(path, "w") as f:
        for row in np.asarray(matrix):
            f.write(" ".join(str(int(v)) for v in row) + " \n")


# ----------------------------------------------------------------------------------------------
# synthetic inputs (seeded) with the shapes of the benchmark configurations
# ----------------------------------------------------------------------------------------------

def exponential_mu_distribution(n_fibers: int, n_mus: int, seed: int) -> np.ndarray:
    """Fiber -> motor unit with MU sizes growing exponentially (MU k has weight basis**k), the
    shape of scripts/generate_fiber_distribution.py; motor units are numbered from 1."""
    rng = np.random.default_rng(seed)
    basis = 1.0 + 3.0 / max(n_mus, 1)  # the largest MU is ~20x the smallest for 100 MUs
    w = basis ** np.arange(n_mus)
    w /= w.sum()
    return rng.choice(np.arange(1, n_mus + 1), size=n_fibers, p=w).astype(np.int32)


def poisson_firing_times(n_mus: int, t_end_ms: float, frequency_per_ms: float, rate_hz_low: float,
                         rate_hz_high: float, seed: int) -> np.ndarray:
    """Rows = sampling steps at ``frequency_per_ms`` (the setSpecificStatesCallFrequency), columns =
    motor units; each MU fires as a Poisson process with a rate drawn from U[low, high] Hz
    (cf. scripts/generate_firing_times.py).  Column 0 is unused by MU numbers starting at 1 and is
    a copy of column 1."""
    rng = np.random.default_rng(seed)
    n_rows = int(math.ceil(t_end_ms * frequency_per_ms)) + 1
    rates = rng.uniform(rate_hz_low, rate_hz_high, size=n_mus) * 1e-3  # per ms
    p = 1.0 - np.exp(-rates / frequency_per_ms)
    fire = (rng.random((n_rows, n_mus)) < p[None, :]).astype(np.uint8)
    out = np.zeros((n_rows, n_mus + 1), np.uint8)
    out[:, 1:] = fire
    out[:, 0] = fire[:, 0]
    return out
