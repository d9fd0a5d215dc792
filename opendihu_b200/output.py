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
import warnings
from typing import Callable, Dict, List, Optional, Sequence

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


class OutputWriter:
    """One entry of an ``"OutputWriter"`` settings list of the diffusion solver, for the fibers it covers.

    When it writes restates ``OutputWriter::Generic::prepareWrite`` (core/src/output_writer/generic.tpp:14-115):
    every call adds ``callCountIncrement`` to a call counter; a file is due when the counter passes a multiple
    of ``outputInterval`` (``generic.cpp:20``, default 1), or when the increment is 0 (initial values).  Its
    name is ``<filename>_<no:07d>`` with ``no`` the running file number (``"fileNumbering": "incremental"``,
    the default) or the call counter (``"timeStepIndex"``).  Formats: ``PythonFile`` writes ``<name>.py``
    (``<name>_<meshName>.py`` for a writer over several fibers, python_file.tpp:30-43) as JSON text, or as a
    pickle with ``"binary": True`` (python_file.tpp:72); ``PythonCallback`` calls ``callback(list of the fiber
    dicts)`` (python_callback_writer.tpp:68).  Other formats (Paraview, Exfile, MegaMol) are not built: they
    warn once and write nothing.
    """

    FORMATS = ("PythonFile", "PythonCallback")

    def __init__(self, settings: dict, fibers: Sequence[int], mesh_names: Optional[Sequence[str]] = None):
        self.format = str(settings.get("format", "none"))
        try:
            interval = int(settings.get("outputInterval", 1))
        except (TypeError, ValueError):
            interval = 1
        self.output_interval = interval if interval > 0 else 1
        self.filename = str(settings.get("filename", "out"))
        self.file_numbering = "timeStepIndex" if settings.get("fileNumbering") == "timeStepIndex" else "incremental"
        self.binary = bool(settings.get("binary", False))
        self.callback: Optional[Callable] = settings.get("callback")
        self.fibers = [int(f) for f in fibers]
        self.mesh_names = list(mesh_names) if mesh_names is not None else [f"MeshFiber_{f}" for f in self.fibers]
        self.write_call_count = 0
        self.output_file_no = 0
        if self.format not in self.FORMATS:
            warnings.warn(f"OutputWriter format {self.format!r} is not built (PythonFile and PythonCallback are); "
                          f"nothing is written for it")
        elif self.format == "PythonCallback" and not callable(self.callback):
            raise ValueError("OutputWriter: format PythonCallback needs a callable 'callback'")

    def prepare(self, time_step_no: int, current_time: float, call_count_increment: int = 1) -> Optional[str]:
        """Counts one call; the numbered file name base when this call writes, else None."""
        old = self.write_call_count
        self.write_call_count += int(call_count_increment)
        last = self.write_call_count - self.write_call_count % self.output_interval
        if not ((old < last <= self.write_call_count) or call_count_increment == 0):
            return None
        name = self.filename
        if time_step_no != -1:
            no = self.output_file_no if self.file_numbering == "incremental" else self.write_call_count
            name += f"_{no:07d}"
        self.output_file_no += 1
        return name

    def write(self, name: str, dicts: Sequence[dict]) -> List[str]:
        """Writes the fiber dicts (one per covered fiber, in order) under ``name``; the paths written."""
        if self.format == "PythonCallback":
            self.callback(list(dicts))
            return []
        if self.format != "PythonFile":
            return []
        d = os.path.dirname(name)
        if d:
            os.makedirs(d, exist_ok=True)
        paths = []
        for mesh, data in zip(self.mesh_names, dicts):
            path = f"{name}.py" if len(dicts) == 1 else f"{name}_{mesh}.py"
            if self.binary:
                with open(path, "wb") as fh:
                    pickle.dump(data, fh, 1)
            else:
                with open(path, "w") as fh:
                    json.dump(data, fh)
            paths.append(path)
        return paths


def write_stimulation_log(filename: str, times, fibers, motor_units) -> None:
    """The stimulation log file of the reference's StimulationLogging::writeLogFile
    (core/src/control/diagnostic_tool/stimulation_logging.cpp:119-165): entries sorted by motor unit, then fiber,
    then time; a header line, then one line ``<motor unit>;<fiber>;<t1>;<t2>;...;`` per (motor unit, fiber), the
    times as a C++ stream writes a double (6 significant digits), no newline after the last line.  Nothing is
    written for an empty log, as in the reference."""
    t = np.asarray(times, np.float64)
    f = np.asarray(fibers, np.int64)
    m = np.asarray(motor_units, np.int64)
    if len(t) == 0:
        return
    order = np.lexsort((t, f, m))
    d = os.path.dirname(filename)
    if d:
        os.makedirs(d, exist_ok=True)
    lines = []
    cur = None
    for i in order:
        key = (int(m[i]), int(f[i]))
        if key != cur:
            cur = key
            lines.append(f"{key[0]};{key[1]};")
        lines[-1] += f"{float(t[i]):g};"
    with open(filename, "w") as fh:
        fh.write("# motor unit no; fiber no; stimulation times in ms\n" + "\n".join(lines))
