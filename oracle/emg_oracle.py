"""CPU oracle of the fibers -> 3D static bidomain (EMG) chain -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline may import this module; the
product path (opendihu_b200.emg over libfdm_b200.so) never does.

A plain numpy / scipy restatement of the reference's algorithms, each function naming the reference code it
follows:
  * trilinear hexahedral elements, dof order a + 2b + 4c (x fastest) as the reference's
    StructuredDeformableOfDimension<3> with LagrangeOfOrder<1>;
  * stiffness matrices int grad(phi_l) . sigma . grad(phi_m) with tensor-product Gauss-Legendre quadrature
    (numpy's ``leggauss``), assembled into a scipy sparse matrix;
  * the directional tensor rotation of math_utility.tpp:587-655 (rotateMatrix, both branches with the
    reference's formulas) applied to the interpolated nodal direction (diffusion_tensor_directional.tpp:72-110);
  * the potential flow with Dirichlet values and its nodal gradient field
    (static_bidomain_solver.tpp:102-130, 08_field_variable_gradient.tpp:59-115);
  * the fiber -> mesh mapping (mapping_between_meshes 00_construct.tpp:90-160, 01_implementation.tpp:15-60,
    03_manager_implementation.tpp:239-300) with a brute-force element search (lowest element index among the
    elements containing the point; else the element whose xi leaves [0,1] least, accepted within xiTolerance);
  * the static bidomain solve K(sigma_i + sigma_e) phi_e = -K(sigma_i) Vm (static_bidomain_solver.tpp:37-55),
    solved directly (one node pinned, then the mean removed: the zero-mean solution).
Parity is pinned to analytic cases (the unit-cube Laplace element matrix, exact linear potential flows,
sigma_e = 0 giving phi_e = -(Vm - mean Vm)); the reference's PETSc path itself is not run here.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def box_mesh(n_nodes, extent, offset=(0.0, 0.0, 0.0)):
    """Node positions [N, 3] of an axis-aligned box with n_nodes = (nx, ny, nz), x fastest."""
    nx, ny, nz = n_nodes
    xs = [offset[d] + np.linspace(0.0, extent[d], n) for d, n in enumerate(n_nodes)]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def element_nodes(shape):
    """[E, 8] node numbers of the elements (element (ex, ey, ez) numbered ex + (nx-1)(ey + (ny-1) ez))."""
    nx, ny, nz = shape
    ex, ey, ez = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1), indexing="ij")
    ex, ey, ez = (a.transpose(2, 1, 0).ravel() for a in (ex, ey, ez))
    out = np.empty((len(ex), 8), np.int64)
    for l in range(8):
        a, b, c = l & 1, (l >> 1) & 1, l >> 2
        out[:, l] = (ex + a) + nx * ((ey + b) + ny * (ez + c))
    return out


def shape_functions(xi):
    """phi [..., 8] and dphi/dxi [..., 8, 3] at xi [..., 3]."""
    xi = np.asarray(xi, float)
    phi = np.empty(xi.shape[:-1] + (8,))
    dphi = np.empty(xi.shape[:-1] + (8, 3))
    for l in range(8):
        s = [(l >> d) & 1 for d in range(3)]
        f = [xi[..., d] if s[d] else 1.0 - xi[..., d] for d in range(3)]
        g = [1.0 if s[d] else -1.0 for d in range(3)]
        phi[..., l] = f[0] * f[1] * f[2]
        dphi[..., l, 0] = g[0] * f[1] * f[2]
        dphi[..., l, 1] = f[0] * g[1] * f[2]
        dphi[..., l, 2] = f[0] * f[1] * g[2]
    return phi, dphi


def rotate_tensor(S, b):
    """math_utility.tpp:587-655 (rotateMatrix): S given in fiber coordinates, first axis onto b."""
    b1, b2, b3 = b
    bn = np.sqrt(b1 * b1 + b2 * b2 + b3 * b3)
    e3b = np.sqrt(b1 * b1 + b2 * b2)
    be3b = np.sqrt(b1 * b1 * b3 * b3 + b2 * b2 * b3 * b3 + (b1 * b1 + b2 * b2) ** 2)
    if abs(bn) < 1e-15:
        return S
    if abs(e3b) < 1e-15 or abs(be3b) < 1e-15:
        e2b = np.sqrt(b3 * b3 + b1 * b1)
        be2b = np.sqrt(b1 * b1 * b2 * b2 + (b1 * b1 * b3 * b3) ** 2 + b2 * b2 + b3 * b3)
        if abs(e2b) < 1e-15 or abs(be2b) < 1e-15:
            return S
        B = np.array([[b1 / bn, b3 / e2b, -b1 * b2 / be2b],
                      [b2 / bn, 0.0, (b1 * b1 + b3 * b3) / be2b],
                      [b3 / bn, -b1 / e2b, -b2 * b3 / be2b]])
    else:
        B = np.array([[b1 / bn, -b2 / e3b, -b1 * b3 / be3b],
                      [b2 / bn, b1 / e3b, -b2 * b3 / be3b],
                      [b3 / bn, 0.0, (b1 * b1 + b2 * b2) / be3b]])
    return B @ S @ B.T


def stiffness(pos, shape, tensors, gauss, direction=None, tensors2=None, prefactor=1.0):
    """Sparse K with K[m, l] = prefactor int grad(phi_l) . sigma . grad(phi_m) over all elements.
    tensors: [1 or E, 3, 3] (plus tensors2, added before the rotation); direction [N, 3] or None."""
    pts, wts = np.polynomial.legendre.leggauss(gauss)
    pts = 0.5 * (pts + 1.0)
    wts = 0.5 * wts
    en = element_nodes(shape)
    E = len(en)
    T1 = np.asarray(tensors, float).reshape(-1, 3, 3)
    T2 = None if tensors2 is None else np.asarray(tensors2, float).reshape(-1, 3, 3)
    rows, cols, vals = [], [], []
    qxi = np.array([[pts[i], pts[j], pts[k]] for k in range(gauss) for j in range(gauss) for i in range(gauss)])
    qw = np.array([wts[i] * wts[j] * wts[k] for k in range(gauss) for j in range(gauss) for i in range(gauss)])
    phi, dphi = shape_functions(qxi)
    for e in range(E):
        P = pos[en[e]]                                       # [8, 3]
        J = np.einsum("li,qld->qid", P, dphi)                # [Q, 3, 3] dx_i/dxi_d
        det = np.linalg.det(J)
        inv = np.linalg.inv(J)                               # dxi_d/dx_i as inv[q, d, i]
        G = np.einsum("qdi,qld->qli", inv, dphi)             # world gradients [Q, 8, 3]
        S0 = T1[0 if len(T1) == 1 else e] + (0.0 if T2 is None else T2[0 if len(T2) == 1 else e])
        Ke = np.zeros((8, 8))
        for q in range(len(qw)):
            S = S0
            if direction is not None:
                b = phi[q] @ direction[en[e]]
                if not np.all(np.isfinite(b)):
                    b = np.array([0.0, 0.0, 1.0])
                S = rotate_tensor(S0, b)
            Ke += prefactor * qw[q] * abs(det[q]) * (G[q] @ S @ G[q].T)
        rows.append(np.repeat(en[e], 8))
        cols.append(np.tile(en[e], 8))
        vals.append(Ke.ravel())
    N = len(pos)
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))


def potential_flow(pos, shape, dirichlet_nodes, dirichlet_values, gauss=3):
    """Laplace with Dirichlet values, solved directly; returns (u, nodal direction [N, 3])."""
    K = stiffness(pos, shape, np.eye(3), gauss).tocsr()
    N = len(pos)
    d = np.asarray(dirichlet_nodes, np.int64)
    free = np.ones(N, bool)
    free[d] = False
    u = np.zeros(N)
    u[d] = dirichlet_values
    Kff = K[free][:, free]
    rhs = -(K[free][:, ~free] @ u[~free])
    u[free] = spla.spsolve(Kff.tocsc(), rhs)
    return u, gradient_direction(pos, shape, u)


def gradient_direction(pos, shape, u):
    """08_field_variable_gradient.tpp:59-115: per element and corner, the gradient at the corner divided by the
    node's number of adjacent elements, summed into the node; then normalised."""
    en = element_nodes(shape)
    N = len(pos)
    n_adj = np.bincount(en.ravel(), minlength=N)
    grad = np.zeros((N, 3))
    corners = np.array([[l & 1, (l >> 1) & 1, l >> 2] for l in range(8)], float)
    _, dphi = shape_functions(corners)                      # [8 corners, 8, 3]
    for e in range(len(en)):
        P = pos[en[e]]
        for c in range(8):
            J = P.T @ dphi[c]                                # [3, 3]
            gxi = u[en[e]] @ dphi[c]
            gw = np.linalg.inv(J).T @ gxi
            grad[en[e][c]] += gw / n_adj[en[e][c]]
    with np.errstate(invalid="ignore", divide="ignore"):
        return grad / np.linalg.norm(grad, axis=1)[:, None]


def _locate(P, x):
    """xi of x in the element with corner positions P [8, 3] (Newton on the trilinear map)."""
    xi = np.full(3, 0.5)
    for _ in range(50):
        phi, dphi = shape_functions(xi)
        r = phi @ P - x
        J = P.T @ dphi
        dx = np.linalg.solve(J, r)
        xi = xi - dx
        if not np.max(np.abs(dx)) > 1e-15:
            break
    return xi, max(0.0, float(np.max(np.maximum(-xi, xi - 1.0))))


def fiber_mapping(pos, shape, points, xi_tolerance=0.1, default_value=0.0):
    """Per fiber node the element and the 8 factors (or None outside); returns (elements, factors, mapped)."""
    if xi_tolerance <= 0:
        xi_tolerance = 0.1
    en = element_nodes(shape)
    lo = pos[en].min(axis=1)
    hi = pos[en].max(axis=1)
    elems, facs = [], []
    for x in np.asarray(points, float):
        cand = np.nonzero(np.all((x >= lo - 1e-9) & (x <= hi + 1e-9), axis=1))[0]
        best_e, best_o, best_xi = -1, np.inf, None
        for e in cand:                                      # lowest index containing the point
            xi, o = _locate(pos[en[e]], x)
            if o <= 1e-12:
                best_e, best_o, best_xi = e, o, xi
                break
            if o < best_o:
                best_e, best_o, best_xi = e, o, xi
        if best_e < 0 or best_o > 1e-12:
            for e in range(len(en)):                        # not inside any bounding box: least violation
                xi, o = _locate(pos[en[e]], x)
                if o < best_o - 1e-15:
                    best_e, best_o, best_xi = e, o, xi
        if best_o > xi_tolerance:
            elems.append(-1)
            facs.append(None)
            continue
        phi, _ = shape_functions(best_xi)
        phi = np.where(np.abs(phi) < 1e-14, np.where(phi >= 0, 1e-14, -1e-14), phi)
        elems.append(best_e)
        facs.append(phi)
    return np.array(elems), facs


def map_values(pos, shape, elems, facs, values, default_value=0.0):
    """Vm on the 3D nodes: sum of factor * value over the fiber nodes (in fiber-node order), divided by the
    factor sum (|sum| <= 1e-12: default_value)."""
    en = element_nodes(shape)
    N = len(pos)
    acc = np.zeros(N)
    fsum = np.zeros(N)
    for s, e in enumerate(elems):
        if e < 0:
            continue
        for l in range(8):
            acc[en[e][l]] += facs[s][l] * values[s]
            fsum[en[e][l]] += facs[s][l]
    out = np.full(N, float(default_value))
    ok = np.abs(fsum) > 1e-12
    out[ok] = acc[ok] / fsum[ok]
    return out


def bidomain(K_i, K_ie, vm):
    """phi_e of K_ie phi_e = -K_i vm (constants as null space): node 0 pinned, then the mean removed."""
    rhs = -(K_i @ vm)
    A = K_ie.tocsr()[1:, 1:].tocsc()
    phi = np.zeros(len(vm))
    phi[1:] = spla.spsolve(A, rhs[1:])
    return phi - phi.mean(), rhs


def stencil_to_sparse(coef, shape):
    """The library's 27-point stencil coef[27, N] as a scipy matrix (for comparisons)."""
    nx, ny, nz = shape
    N = nx * ny * nz
    n = np.arange(N)
    i, j, k = n % nx, (n // nx) % ny, n // (nx * ny)
    rows, cols, vals = [], [], []
    for q in range(27):
        dx, dy, dz = q % 3 - 1, (q // 3) % 3 - 1, q // 9 - 1
        ok = (i + dx >= 0) & (i + dx < nx) & (j + dy >= 0) & (j + dy < ny) & (k + dz >= 0) & (k + dz < nz)
        rows.append(n[ok])
        cols.append(n[ok] + dx + nx * (dy + ny * dz))
        vals.append(coef[q][ok])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
