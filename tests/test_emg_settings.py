"""EMG host logic without a device: 3D meshes from settings, Dirichlet values with negative node numbers,
tensor lists, fiber node positions, the Coupling's step count and its refusal of transfers other than Vm."""
import numpy as np
import pytest

import test_gpu_emg as GE
from opendihu_b200 import emg as E


def test_mesh_from_settings():
    shape, pos = E.mesh_from_settings({"nElements": [2, 3, 4], "physicalExtent": [1.0, 1.5, 2.0],
                                       "physicalOffset": [0.5, 0.0, -1.0]})
    assert shape == (3, 4, 5) and pos.shape == (60, 3)
    np.testing.assert_allclose(pos[0], [0.5, 0.0, -1.0])
    np.testing.assert_allclose(pos[1], [1.0, 0.0, -1.0])          # x fastest
    np.testing.assert_allclose(pos[-1], [1.5, 1.5, 1.0])
    shape2, pos2 = E.mesh_from_settings({"nElements": [2, 3, 4], "nodePositions": pos.tolist()})
    assert shape2 == shape
    np.testing.assert_array_equal(pos2, pos)
    with pytest.raises(ValueError):
        E.mesh_from_settings({"nElements": [2, 3, 4], "nodePositions": pos[:-1].tolist()})


def test_dirichlet_and_tensors():
    nodes, vals = E._dirichlet({0: 0.0, -1: 1.0, 3: [2.0], 5: None}, 10)
    np.testing.assert_array_equal(nodes, [0, 9, 3])
    np.testing.assert_array_equal(vals, [0.0, 1.0, 2.0])
    assert E._tensors([[1, 0, 0, 0, 2, 0, 0, 0, 3]], 7).shape == (1, 9)
    assert E._tensors(np.ones((7, 9)), 7).shape == (7, 9)
    with pytest.raises(ValueError):
        E._tensors(np.ones((3, 9)), 7)


def test_fiber_positions_from_settings():
    meshes = {"a": {"nElements": [2], "nodePositions": [[0, 0, 0], [0, 0, 1], [0, 0, 2]]},
              "b": {"nElements": [4], "physicalExtent": [2.0], "physicalOffset": [1.0, 2.0]}}
    p = E.fiber_positions_from_settings(meshes, ["a", "b"])
    assert p.shape == (8, 3)
    np.testing.assert_allclose(p[3:], [[1.0, 2.0, 0.0], [1.5, 2.0, 0.0], [2.0, 2.0, 0.0], [2.5, 2.0, 0.0],
                                       [3.0, 2.0, 0.0]])


def test_coupling_from_settings_on_the_host():
    cfg, fpos, kw = GE._settings()
    cp = E.Coupling.from_settings(cfg)           # nothing touches the device before initialize()
    assert cp.n_time_steps() == 2 and cp.time_step_width == 0.5
    np.testing.assert_allclose(cp.fiber_positions, fpos)
    assert cp.term2.shape == kw["shape"]
    np.testing.assert_array_equal(np.sort(cp.term2.dirichlet_nodes), np.sort(kw["dirichlet_nodes"]))
    assert cp.term2.emg_solver["relativeTolerance"] == GE.TIGHT["relativeTolerance"]
    cfg["Coupling"]["connectedSlotsTerm1To2"] = {1: 0}
    with pytest.raises(ValueError):
        E.Coupling.from_settings(cfg)


def test_bidomain_needs_directions_or_boundary_values():
    _, _, kw = GE._settings()
    with pytest.raises(ValueError):
        E.StaticBidomainSolver(kw["shape"], kw["node_positions"], kw["sigma_i"], kw["sigma_e"])
