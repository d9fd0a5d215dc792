"""Fibers -> 3D static bidomain (EMG) on the GPU against the oracle (oracle/emg_oracle.py): the potential flow
and fiber directions on a deformed mesh, the assembled stencils (one tensor for all elements and one per
element), the fiber -> mesh transfer (host values and straight from the fiber solver's device Vm), phi_e,
phi_e = -(Vm - mean Vm) without extracellular conduction at a larger size, and the Coupling driven from a
reference-shaped settings dict against the oracles of both solvers."""
import numpy as np
import pytest

import helpers as H
from oracle import emg_oracle as EO
from opendihu_b200 import emg as E
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL

pytestmark = pytest.mark.gpu

TIGHT = {"relativeTolerance": 1e-13, "absoluteTolerance": 1e-30, "maxIterations": 20000}


def _deformed_mesh(shape=(6, 5, 9), ext=(1.0, 0.8, 2.0), seed=3):
    rng = np.random.default_rng(seed)
    pos = EO.box_mesh(shape, ext)
    # a smooth bend (the fibers' direction varies) plus small random jitter
    pos[:, 0] += 0.15 * np.sin(pos[:, 2] / ext[2] * np.pi)
    pos += rng.uniform(-0.02, 0.02, size=pos.shape)
    nx, ny, nz = shape
    lo = np.arange(nx * ny)
    hi = lo + nx * ny * (nz - 1)
    return shape, pos, np.concatenate([lo, hi]), np.r_[np.zeros(nx * ny), np.ones(nx * ny)]


def _solver(shape, pos, bn, bv, **kw):
    kw.setdefault("sigma_i", WL.EMG_SIGMA_I)
    kw.setdefault("sigma_e", WL.EMG_SIGMA_E)
    return E.StaticBidomainSolver(shape, pos, dirichlet_nodes=bn, dirichlet_values=bv,
                                  potential_flow_solver=TIGHT, emg_solver=TIGHT, **kw)


@pytest.mark.parametrize("per_element", [False, True])
def test_potential_flow_stencils_and_phi_match_oracle(per_element):
    shape, pos, bn, bv = _deformed_mesh()
    ne = (shape[0] - 1) * (shape[1] - 1) * (shape[2] - 1)
    rng = np.random.default_rng(4)
    si = np.asarray(WL.EMG_SIGMA_I, float).reshape(3, 3)
    se = np.asarray(WL.EMG_SIGMA_E, float).reshape(3, 3)
    if per_element:
        si = si[None] * rng.uniform(0.5, 1.5, size=(ne, 1, 1))
        se = se[None] * rng.uniform(0.5, 1.5, size=(ne, 1, 1))
    u_ref, d_ref = EO.potential_flow(pos, shape, bn, bv, gauss=3)
    Ki = EO.stiffness(pos, shape, si, 5, direction=d_ref)
    Kie = EO.stiffness(pos, shape, si, 5, direction=d_ref, tensors2=se)
    vm = rng.normal(-70.0, 20.0, size=len(pos))
    phi_ref, rhs_ref = EO.bidomain(Ki, Kie, vm)
    with _solver(shape, pos, bn, bv, sigma_i=si.reshape(-1, 9), sigma_e=se.reshape(-1, 9)) as slv:
        np.testing.assert_allclose(slv.flow_potential(), u_ref, rtol=0, atol=1e-11)
        np.testing.assert_allclose(slv.fiber_direction(), d_ref, rtol=0, atol=1e-10)
        for which, K in ((0, Ki), (1, Kie)):
            got = EO.stencil_to_sparse(slv.stencil(which), shape)
            assert abs(got - K).max() <= 1e-9 * abs(K).max()
        slv.set_vm(vm)
        its = slv.advanceTimeSpan()
        assert its > 0
        np.testing.assert_allclose(slv.rhs(), rhs_ref, rtol=0, atol=1e-8 * np.abs(rhs_ref).max())
        phi = slv.phi_e()
    assert abs(phi.mean()) < 1e-10
    np.testing.assert_allclose(phi, phi_ref, rtol=0, atol=1e-8 * np.abs(phi_ref).max())


def test_mapping_matches_oracle_and_device_transfer():
    s, fpos, kw = WL.emg_box(n_fibers_x=3, n_fibers_y=2, n_nodes=61, mesh_nodes=(4, 3, 7), width=1.0, end_time=0.3)
    fpos = fpos.copy()
    fpos[5] = [9.0, 9.0, 9.0]                       # one fiber node outside the mesh
    el, fac = EO.fiber_mapping(kw["node_positions"], kw["shape"], fpos)
    vals = np.random.default_rng(5).normal(size=len(fpos))
    want = EO.map_values(kw["node_positions"], kw["shape"], el, fac, vals, default_value=-7.0)
    with E.StaticBidomainSolver(**kw) as slv:
        assert slv.set_fiber_mapping(fpos, default_value=-7.0) == len(fpos) - 1
        slv.map_values(vals)
        np.testing.assert_allclose(slv.vm(), want, rtol=0, atol=1e-12)
        # straight from the fiber solver's device Vm, after an advance
        with S.FastMonodomainSolver(H.complete(s.copy()), method="fused") as fib:
            fib.advanceTimeSpan()
            slv.map_fibers(fib)
            got = slv.vm()
            vm_f = fib.states()[0]
        np.testing.assert_allclose(got, EO.map_values(kw["node_positions"], kw["shape"], el, fac, vm_f, -7.0),
                                   rtol=0, atol=1e-12)


def test_no_extracellular_conduction_at_size():
    s, fpos, kw = WL.emg_box(n_fibers_x=2, n_fibers_y=2, n_nodes=101, mesh_nodes=(33, 33, 65), width=1.0)
    kw["sigma_e"] = np.zeros(9)
    rng = np.random.default_rng(6)
    vm = rng.normal(size=33 * 33 * 65)
    with E.StaticBidomainSolver(emg_solver=TIGHT, potential_flow_solver=TIGHT, **kw) as slv:
        np.testing.assert_allclose(slv.fiber_direction(), np.tile([0, 0, 1.0], (33 * 33 * 65, 1)), atol=1e-9)
        slv.set_vm(vm)
        slv.advanceTimeSpan()
        phi = slv.phi_e()
        t = slv.timing()
    np.testing.assert_allclose(phi, -(vm - vm.mean()), rtol=0, atol=1e-7)
    assert t["iterations"] > 0 and t["solve_ms"] > 0


def _settings(n_fx=2, n_fy=2, n_nodes=41, mesh=(4, 4, 6), width=1.0, dt3d=0.5, end=1.0):
    s, fpos, kw = WL.emg_box(n_fibers_x=n_fx, n_fibers_y=n_fy, n_nodes=n_nodes, mesh_nodes=mesh, width=width,
                             end_time=end)
    nf = n_fx * n_fy
    names = [f"MeshFiber_{i}" for i in range(nf)]
    meshes = {n: {"nElements": [n_nodes - 1], "nodePositions": fpos[i * n_nodes:(i + 1) * n_nodes].tolist()}
              for i, n in enumerate(names)}
    nx, ny, nz = mesh
    meshes["3Dmesh"] = {"nElements": [nx - 1, ny - 1, nz - 1], "physicalExtent": [width, width, (n_nodes - 1) * 0.01]}
    heun = [{"Heun": {"timeStepWidth": 1e-4, "CellML": {
        "modelFilename": "hodgkin_huxley_1952.c", "setSpecificStatesCallFrequency": 0.1,
        "setSpecificStatesRepeatAfterFirstCall": 0.1, "setSpecificStatesCallEnableBegin": 0.0,
        "parametersUsedAsAlgebraic": [], "parametersUsedAsConstant": [2, 3, 4],
        "parametersInitialValues": [0.0, 120.0, 36.0], "meshName": n}}} for n in names]
    diff = [{"ImplicitEuler": {"timeStepWidth": 1e-3, "FiniteElementMethod": {
        "meshName": n, "prefactor": WL.SIGMA / (WL.AM * WL.CM)}}} for n in names]
    strang = {"StrangSplitting": {"timeStepWidth": 1e-3, "Term1": {"MultipleInstances": {"instances": heun}},
                                  "Term2": {"MultipleInstances": {"instances": diff}}}}
    bc = {int(k): 0.0 for k in range(nx * ny)}
    bc.update({int(k) - nx * ny: 1.0 for k in range(nx * ny)})      # negative: counted from the end
    fem = {"meshName": "3Dmesh", "prefactor": 1.0, "solverName": "muscularEMGSolver",
           "diffusionTensor": [list(WL.EMG_SIGMA_I)], "extracellularDiffusionTensor": [list(WL.EMG_SIGMA_E)]}
    cfg = {
        "Meshes": meshes,
        "Solvers": {"potentialFlowSolver": TIGHT, "muscularEMGSolver": TIGHT},
        "MappingsBetweenMeshes": {n: ["3Dmesh"] for n in names},
        "Coupling": {
            "timeStepWidth": dt3d, "endTime": end, "connectedSlotsTerm1To2": {0: 0}, "connectedSlotsTerm2To1": [None],
            "Term1": {"MultipleInstances": {"instances": [strang]}, "onlyComputeIfHasBeenStimulated": False,
                      "disableComputationWhenStatesAreCloseToEquilibrium": False},
            "Term2": {"StaticBidomainSolver": {
                "timeStepWidth": dt3d, "solverName": "muscularEMGSolver", "initialGuessNonzero": True,
                "PotentialFlow": {"FiniteElementMethod": {"meshName": "3Dmesh", "solverName": "potentialFlowSolver",
                                                          "prefactor": 1.0, "dirichletBoundaryConditions": bc}},
                "Activation": {"FiniteElementMethod": fem}}},
        },
    }
    return cfg, fpos, kw


def test_coupling_from_settings_matches_oracles():
    cfg, fpos, kw = _settings()
    phis = []
    cp = E.Coupling.from_settings(cfg)
    cp.callback = lambda k, t, emg: phis.append((t, emg.phi_e()))
    with cp:
        assert cp.n_mapped == len(fpos)
        cp.run()
        system = cp.term1.system
    assert [round(t, 9) for t, _ in phis] == [0.5, 1.0]
    # oracle chain: fibers to 0.5 and 1.0 ms, mapped, bidomain
    shape, pos = kw["shape"], kw["node_positions"]
    u, d = EO.potential_flow(pos, shape, kw["dirichlet_nodes"], kw["dirichlet_values"], gauss=3)
    si = np.asarray(WL.EMG_SIGMA_I).reshape(3, 3)
    Ki = EO.stiffness(pos, shape, si, 5, direction=d)
    Kie = EO.stiffness(pos, shape, si, 5, direction=d, tensors2=np.asarray(WL.EMG_SIGMA_E).reshape(3, 3))
    el, fac = EO.fiber_mapping(pos, shape, fpos)
    sysc = H.complete(system.copy())
    run = H.O.OracleRun(H.oracle_spec(sysc.copy()))
    st = np.ascontiguousarray(sysc.states, np.float64).copy()
    for (t, phi), (a, b) in zip(phis, [(0.0, 0.5), (0.5, 1.0)]):
        run.run(st, a, b)
        want, _ = EO.bidomain(Ki, Kie, EO.map_values(pos, shape, el, fac, st[0]))
        assert np.max(np.abs(phi - want)) <= 1e-6 * max(np.abs(want).max(), 1.0)
    assert np.abs(phis[-1][1]).max() > 0


def test_surface_sample_and_bad_inputs():
    shape, pos, bn, bv = _deformed_mesh()
    rng = np.random.default_rng(9)
    with _solver(shape, pos, bn, bv) as slv:
        slv.set_vm(rng.normal(size=len(pos)))
        slv.advanceTimeSpan()
        phi = slv.phi_e()
        nx, ny, nz = shape
        top = slv.surface("2+")
        assert top.shape == (ny, nx)
        np.testing.assert_array_equal(top, phi[-nx * ny:].reshape(ny, nx))
        np.testing.assert_array_equal(slv.surface("0-"), phi.reshape(nz, ny, nx)[:, :, 0])
        # at nodes the interpolation returns the nodal values; outside the mesh NaN
        pick = [0, 17, len(pos) // 2, len(pos) - 1]
        np.testing.assert_allclose(slv.sample(pos[pick]), phi[pick], rtol=0, atol=1e-9)
        assert np.isnan(slv.sample([[50.0, 50.0, 50.0]]))[0]
        with pytest.raises(S.N.FdmError):
            slv.set_fiber_mapping(np.zeros((3, 3)))
            with S.FastMonodomainSolver(H.complete(H.c1_system(n_fibers=1, n_nodes=11, end_time=0.01))) as f:
                f.initialize()
                slv.map_fibers(f)                # 11 fiber nodes against a mapping of 3
    inverted = pos.copy()
    inverted[:, 0] *= -1.0                       # mirrored: every element inverted
    with pytest.raises(S.N.FdmError) as e:
        E.StaticBidomainSolver(shape, inverted, WL.EMG_SIGMA_I, WL.EMG_SIGMA_E, dirichlet_nodes=bn,
                               dirichlet_values=bv).initialize()
    assert e.value.code == S.N.FDM_ERR_ARG


def test_overlapped_coupling_equals_sequential():
    cfg, fpos, kw = _settings(end=1.5)
    out = {}
    for overlap in (False, True):
        phis = []
        cp = E.Coupling.from_settings(cfg)
        cp.overlap = overlap
        cp.callback = lambda k, t, emg: phis.append((k, round(t, 9), emg.phi_e(), emg.vm()))
        with cp:
            cp.run()
            vm = cp.term1.states()[0]
        out[overlap] = (phis, vm)
    a, b = out[False], out[True]
    np.testing.assert_array_equal(a[1], b[1])
    assert [p[:2] for p in a[0]] == [p[:2] for p in b[0]] == [(0, 0.5), (1, 1.0), (2, 1.5)]
    for pa, pb in zip(a[0], b[0]):
        np.testing.assert_array_equal(pa[2], pb[2])
        np.testing.assert_array_equal(pa[3], pb[3])


@pytest.mark.parametrize("mesh", [(17, 13, 41), (33, 33, 65)])
def test_multigrid_preconditioner_same_solution_fewer_iterations(mesh):
    s, fpos, kw = WL.emg_box(n_fibers_x=2, n_fibers_y=2, n_nodes=101, mesh_nodes=mesh, width=1.0)
    z = kw["node_positions"][:, 2]
    vm = -75.0 + 100.0 * np.exp(-((z - z.mean()) / 0.1) ** 2) + np.random.default_rng(3).normal(size=len(z))
    out = {}
    for pc in ("jacobi", "multigrid"):
        with E.StaticBidomainSolver(emg_solver=TIGHT, potential_flow_solver=TIGHT, preconditioner=pc, **kw) as slv:
            slv.set_vm(vm)
            its = slv.advanceTimeSpan()
            out[pc] = (slv.phi_e(), its, slv.multigrid_levels)
    assert out["multigrid"][2] > 1 and out["jacobi"][2] == 1
    assert out["multigrid"][1] * 3 < out["jacobi"][1], (out["multigrid"][1], out["jacobi"][1])
    ref = out["jacobi"][0]
    np.testing.assert_allclose(out["multigrid"][0], ref, rtol=0, atol=1e-8 * np.abs(ref).max())
