"""The EMG oracle (oracle/emg_oracle.py) against analytic cases: the unit-cube Laplace element matrix, the
rotation of a fiber-coordinate tensor onto a direction, exact linear potential flows and their directions,
phi_e = -(Vm - mean Vm) when sigma_e vanishes, and the mapping's factor normalisation."""
import numpy as np
import pytest

from oracle import emg_oracle as EO


def test_unit_cube_laplace_element():
    pos = EO.box_mesh((2, 2, 2), (1.0, 1.0, 1.0))
    K = EO.stiffness(pos, (2, 2, 2), np.eye(3), gauss=2).toarray()
    for l in range(8):
        for m in range(8):
            differ = bin(l ^ m).count("1")
            want = {0: 1 / 3, 1: 0.0, 2: -1 / 12, 3: -1 / 12}[differ]
            assert abs(K[l, m] - want) < 1e-15
    # quadrature of higher order changes nothing for a constant tensor on a box
    np.testing.assert_allclose(EO.stiffness(pos, (2, 2, 2), np.eye(3), gauss=5).toarray(), K, atol=1e-15)


@pytest.mark.parametrize("b", [(0.0, 0.0, 1.0), (1.0, 0.0, 0.0), (0.3, -0.4, 0.866), (0.0, 0.6, -0.8)])
def test_rotation_puts_the_first_axis_on_the_direction(b):
    b = np.asarray(b) / np.linalg.norm(b)
    S = np.diag([8.93, 0.893, 0.893])
    R = EO.rotate_tensor(S, b)
    np.testing.assert_allclose(R, R.T, atol=1e-14)
    np.testing.assert_allclose(R @ b, 8.93 * b, atol=1e-13)
    np.testing.assert_allclose(np.sort(np.linalg.eigvalsh(R)), [0.893, 0.893, 8.93], atol=1e-13)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_potential_flow_on_a_box_is_linear(axis):
    shape = (4, 5, 6)
    ext = (1.0, 1.5, 2.0)
    pos = EO.box_mesh(shape, ext)
    lo = np.nonzero(np.isclose(pos[:, axis], 0.0))[0]
    hi = np.nonzero(np.isclose(pos[:, axis], ext[axis]))[0]
    u, d = EO.potential_flow(pos, shape, np.concatenate([lo, hi]), np.r_[np.zeros(len(lo)), np.ones(len(hi))])
    np.testing.assert_allclose(u, pos[:, axis] / ext[axis], atol=1e-12)
    want = np.zeros(3)
    want[axis] = 1.0
    np.testing.assert_allclose(d, np.tile(want, (len(pos), 1)), atol=1e-12)


def test_no_extracellular_conduction_gives_minus_vm():
    shape = (5, 4, 7)
    rng = np.random.default_rng(1)
    pos = EO.box_mesh(shape, (1.0, 0.8, 1.6)) + rng.uniform(-0.03, 0.03, size=(140, 3))
    d = np.tile([0.0, 0.0, 1.0], (140, 1))
    Ki = EO.stiffness(pos, shape, np.diag([8.93, 0.893, 0.893]), 3, direction=d)
    vm = rng.normal(size=140)
    phi, rhs = EO.bidomain(Ki, Ki, vm)
    np.testing.assert_allclose(phi, -(vm - vm.mean()), atol=1e-10)
    assert abs(rhs.sum()) < 1e-10


def test_mapping_normalises_by_the_factor_sum():
    shape = (3, 3, 4)
    pos = EO.box_mesh(shape, (1.0, 1.0, 1.5))
    rng = np.random.default_rng(2)
    pts = rng.uniform([0, 0, 0], [1, 1, 1.5], size=(40, 3))
    pts = np.vstack([pts, [[5.0, 5.0, 5.0]]])        # outside the mesh
    el, fac = EO.fiber_mapping(pos, shape, pts)
    assert el[-1] == -1 and np.all(el[:-1] >= 0)
    for f in fac[:-1]:
        assert abs(f.sum() - 1.0) < 1e-12
    out = EO.map_values(pos, shape, el, fac, np.full(len(pts), 3.5), default_value=-1.0)
    hit = np.zeros(len(pos), bool)
    for e in el[:-1]:
        hit[EO.element_nodes(shape)[e]] = True
    np.testing.assert_allclose(out[hit], 3.5, atol=1e-12)
    assert np.all(out[~hit] == -1.0)


def test_laplace_3d_matches_the_reference_test():
    # LaplaceTest.StructuredDeformableMatrixIsCorrect3DStencils of the reference (fixture made from its source by
    # tests/golden/make_golden.py): 4 x 4 x 4 trilinear elements of unit size, Gauss quadrature of order 2; the
    # expected matrix is the element stencil summed over the elements, in the reference's sign (-K)
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "laplace3d_golden.json")))
    nx, ny, nz = g["n_elements"]
    shape = (nx + 1, ny + 1, nz + 1)
    st = np.asarray(g["stencil_dy_dx_dz"])
    n = shape[0] * shape[1] * shape[2]
    node = lambda x, y, z: z * shape[0] * shape[1] + y * shape[0] + x
    want = np.zeros((n, n))
    for x in range(nx):
        for y in range(ny):
            for z in range(nz):
                corners = [(x + i, y + j, z + k) for k in (0, 1) for j in (0, 1) for i in (0, 1)]
                for a in corners:
                    for b in corners:
                        want[node(*a), node(*b)] += st[abs(a[1] - b[1]), abs(a[0] - b[0]), abs(a[2] - b[2])]
    pos = EO.box_mesh(shape, g["physical_extent"])
    K = EO.stiffness(pos, shape, np.eye(3), gauss=2).toarray()
    np.testing.assert_allclose(-K, want, rtol=0, atol=g["tolerance"])
