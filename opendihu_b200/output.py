"""PythonFile-compatible output of fiber data.

The reference's PythonFile output writer (core/src/output_writer/python_file/python_file.tpp) writes one
``<filename>_<outputFileNo:07d>.py`` per output step: a dict serialised as JSON text (``"binary": False``)
or as a pickle (``"binary": True``) with the mesh description and one entry per field variable with its
components.  Its readers (testing/unit_testing/src/py_reader.py, the comparison scripts) take those dicts;
this module writes the same layout for each 1D fiber so that they can read the B200 solver's results
(Vm and the other transferred states, per fiber, with the node coordinates as "geometry").
"""
from __future__ import annotations

import json
import os
import pickle
from typing import Dict, Optional, Sequence

import numpy as np


def fiber_dict(values: Dict[str, np.ndarray], geometry: Optional[np.ndarray], time_step_no: int,
               current_time: float, field_name: str = "solution",
               additional: Optional[Dict[str, np.ndarray]] = None) -> dict:
    """The dict of one fiber (StructuredDeformable 1D mesh with linear Lagrange basis); ``additional`` adds
    one single-component field variable per entry (transferred algebraics, computeStateInformation)."""
    n_nodes = len(next(iter(values.values())))
    if geometry is None:
        geometry = np.zeros((n_nodes, 3))
    geometry = np.asarray(geometry, np.float64).reshape(n_nodes, 3)
    return {
        "meshType": "StructuredDeformable", "dimension": 1, "nElementsGlobal": [n_nodes - 1],
        "nElementsLocal": [n_nodes - 1], "beginNodeGlobalNatural": [0], "hasFullNumberOfNodes": [True],
        "basisFunction": "Lagrange", "basisOrder": 1, "onlyNodalValues": True, "nRanks": 1, "ownRankNo": 0,
        "data": [
            {"name": "geometry", "components": [{"name": c, "values": geometry[:, i].tolist()}
                                                for i, c in enumerate("xyz")]},
            {"name": field_name, "components": [{"name": k, "values": np.asarray(v, np.float64).tolist()}
                                                for k, v in values.items()]},
        ] + [{"name": k, "components": [{"name": "0", "values": np.asarray(v, np.float64).tolist()}]}
             for k, v in (additional or {}).items()],
        "timeStepNo": int(time_step_no), "currentTime": float(current_time),
    }


def write_fibers(filename: str, output_no: int, system, states: np.ndarray, state_names: Sequence[str],
                 states_for_transfer: Sequence[int] = (0,), time_step_no: int = 0, current_time: float = 0.0,
                 binary: bool = False, fibers: Optional[Sequence[int]] = None,
                 additional: Optional[Dict[str, np.ndarray]] = None) -> list:
    """Write ``<filename>_<fiber>_<output_no:07d>.py`` for the given fibers (default all) with the chosen
    states; node coordinates are the cumulative element lengths along x; ``additional`` maps field names to
    per-node arrays over all fibers (e.g. "computeStateInformation").  Returns the written paths."""
    off = np.asarray(system.fiber_offsets)
    fibers = range(len(off) - 1) if fibers is None else fibers
    paths = []
    d = os.path.dirname(filename)
    if d:
        os.makedirs(d, exist_ok=True)
    for f in fibers:
        a, b = int(off[f]), int(off[f + 1])
        h = np.asarray(system.element_lengths)[a - f:b - f - 1]
        x = np.concatenate([[0.0], np.cumsum(h)])
        geom = np.stack([x, np.zeros_like(x), np.zeros_like(x)], axis=1)
        vals = {state_names[s]: states[s, a:b] for s in states_for_transfer}
        extra = {k: np.asarray(v)[a:b] for k, v in (additional or {}).items()}
        data = fiber_dict(vals, geom, time_step_no, current_time, additional=extra)
        path = f"{filename}_{f}_{output_no:07d}.py"
        if binary:
            with open(path, "wb") as fh:
                pickle.dump(data, fh, 1)
        else:
            with open(path, "w") as fh:
                json.dump(data, fh)
        paths.append(path)
    return paths


def read(path: str) -> dict:
    """Read one file written by write_fibers (JSON text or pickle), as the reference's readers do."""
    try:
        with open(path) as fh:
            return json.load(fh)
    except (UnicodeDecodeError, json.JSONDecodeError):
        with open(path, "rb") as fh:
            return pickle.load(fh)
