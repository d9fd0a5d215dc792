"""onlyComputeIfHasBeenStimulated on CPU: the library's per-node gate codes (host-only entry point) against a
direct simulation of the reference's buffer-order loop (compute.tpp:158-205), the oracle's behaviour with the
option, and the settings key."""
import numpy as np
import pytest

import helpers as H
from opendihu_b200 import _native as N
from opendihu_b200 import solver as S
from opendihu_b200 import workloads as WL


def _gate_first(code, start):
    """the kernels' rule (fdm_kernels.cuh gate_first) for one node; start: 0 = flag set before the call,
    1 + k = set at substep k, 255 = not set"""
    st = start[code >> 2]
    cls = code & 3
    if st in (0, 255):
        return st
    return st - 1 if cls == 1 else (255 if cls == 0 else 0)


def _reference_first(off, center, W, R, hbs0, kstar):
    """Per node, the first substep the reference computes in one compute0D call: buffers in rank order, the
    junction buffer of the attributed fiber advances its machine (the flag turns on at substep kstar[f]),
    every buffer skips the substeps at which its attributed fiber's flag is still off."""
    n = int(off[-1])
    first = np.full(n, -1)
    for r in range(R):
        fib = list(range(r, len(off) - 1, R))
        if not fib:
            continue
        vo = np.concatenate([[0], np.cumsum([off[f + 1] - off[f] for f in fib])])
        total = vo[-1]
        nbuf = (total + W - 1) // W
        factor = W / (vo[1] - vo[0])
        flag = {f: bool(hbs0[f]) for f in fib}
        for b in range(nbuf):
            local = min(int(b * factor), len(fib) - 1)
            fa = fib[local]
            in_center = 0 <= center[fa] - (b * W - vo[local]) < W
            if flag[fa]:
                fb = 0
            elif in_center and kstar[fa] is not None:
                fb = kstar[fa]
                flag[fa] = True
            else:
                fb = 255
            for lane in range(W):
                i = b * W + lane
                if i >= total:
                    break
                l2 = int(np.searchsorted(vo, i, side="right") - 1)
                first[off[fib[l2]] + i - vo[l2]] = fb
    return first


@pytest.mark.parametrize("W,R,seed", [(4, 1, 0), (4, 2, 1), (8, 3, 2), (1, 1, 3)])
def test_gate_codes_reproduce_the_buffer_order(W, R, seed):
    rng = np.random.default_rng(seed)
    lengths = rng.integers(9, 60, size=11)
    off = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    center = rng.integers(0, lengths).astype(np.int32)
    codes = N.select_gate_codes(S.CLAMP_RULES["vc"], W, R, off, center)
    clamp_first, clamp_cnt, evaluated = N.select_clamp_nodes(S.CLAMP_RULES["vc"], W, R, off, center)
    for trial in range(6):
        hbs0 = rng.integers(0, 2, size=len(lengths)) * (trial % 3 != 0)
        kstar = [int(k) if rng.random() < 0.6 else None for k in rng.integers(0, 5, size=len(lengths))]
        # the machine only runs where a junction buffer exists (the library's "evaluated" flag)
        start = np.array([0 if hbs0[f] else (kstar[f] + 1 if (evaluated[f] and kstar[f] is not None) else 255)
                          for f in range(len(lengths))])
        got = np.array([_gate_first(c, start) for c in codes])
        want = _reference_first(off, center, W, R, hbs0, [k if evaluated[f] else None for f, k in enumerate(kstar)])
        np.testing.assert_array_equal(got, want)


def test_center_rule_gate_codes():
    off = np.array([0, 5, 12], np.int64)
    codes = N.select_gate_codes(S.CLAMP_RULES["center"], 4, 1, off, np.array([2, 3], np.int32))
    np.testing.assert_array_equal(codes, [1] * 5 + [5] * 7)


def _system(only, rule="vc"):
    # three fibers; motor unit 1 never fires, so fiber 1 is never stimulated
    s = WL.batched_hh(n_fibers=3, min_nodes=40, max_nodes=70, seed=5, end_time=0.6, clamp_rule=rule)
    s.firing_events = np.array([[1, 0, 1]], np.uint8)
    s.motor_unit_no = np.array([0, 1, 2], np.int32)
    s.call_enable_begin = np.array([0.0, 0.0, 0.3])
    s.only_compute_if_has_been_stimulated = only
    return H.complete(s)


def test_oracle_skips_fibers_until_stimulated():
    # centre rule (every node follows its own fiber): the never-stimulated fiber 1 stays at rest
    on, _, _, _ = H.run_oracle(_system(True, "center"), n_threads=2)
    off_, _, _, _ = H.run_oracle(_system(False, "center"), n_threads=2)
    s = _system(True, "center")
    o = s.fiber_offsets
    np.testing.assert_allclose(on[:, o[1]:o[2]], s.states[:, o[1]:o[2]], rtol=0, atol=1e-12)
    assert np.max(np.abs(off_[1:, o[1]:o[2]] - s.states[1:, o[1]:o[2]])) > 1e-9
    # vc rule: a point buffer follows the fiber it is attributed to (int(b W / valuesLength[0]), which for
    # uneven lengths can be a neighbouring fiber), so nodes of fiber 1 attributed to a stimulated fiber move
    s = _system(True)
    on, _, _, _ = H.run_oracle(s.copy(), n_threads=2)
    off_, _, _, _ = H.run_oracle(_system(False), n_threads=2)
    codes = N.select_gate_codes(S.CLAMP_RULES["vc"], 4, 1, o, s.stimulation_point_index)
    att = codes >> 2
    never = np.nonzero(att == 1)[0]            # buffers attributed to the never-stimulated fiber
    assert len(never) > 0
    assert np.max(np.abs(on[0] - off_[0])) > 1e-6
    # nodes attributed to fiber 1 are never computed: away from computed neighbours they stay at rest
    quiet = [i for i in never if np.all(att[max(i - 3, 0):i + 4] == 1)]
    np.testing.assert_allclose(on[1:, quiet], s.states[1:, quiet], rtol=0, atol=1e-12)


def reference_settings(n_fibers=2, n_elements=20, **fast):
    """A reference-shaped settings dict (RepeatedCall -> MultipleInstances -> StrangSplitting -> Heun/CellML,
    ImplicitEuler/FiniteElementMethod) for HH fibers of n_elements elements of 0.01 cm."""
    names = [f"MeshFiber_{i}" for i in range(n_fibers)]
    heun = [{"Heun": {"timeStepWidth": 1e-4, "CellML": {
        "modelFilename": "input/hodgkin_huxley_1952.c", "setSpecificStatesCallFrequency": 0.1,
        "setSpecificStatesRepeatAfterFirstCall": 0.1, "setSpecificStatesCallEnableBegin": 0.0,
        "parametersUsedAsAlgebraic": [], "parametersUsedAsConstant": [2, 3, 4],
        "parametersInitialValues": [0.0, 120.0, 36.0], "meshName": n}}} for n in names]
    diff = [{"ImplicitEuler": {"timeStepWidth": 1e-3, "FiniteElementMethod": {"meshName": n, "prefactor": 0.007656}}}
            for n in names]
    strang = {"StrangSplitting": {"timeStepWidth": 1e-3, "Term1": {"MultipleInstances": {"instances": heun}},
                                  "Term2": {"MultipleInstances": {"instances": diff}}}}
    rc = {"timeStepWidth": 1e-3, "endTime": 0.1, "MultipleInstances": {"instances": [strang]}}
    rc.update(fast)
    return {"Meshes": {n: {"nElements": [n_elements], "physicalExtent": [n_elements * 0.01]} for n in names},
            "RepeatedCall": rc}


def test_settings_key():
    s = S.parse_settings(reference_settings())          # the reference's defaults: both True
    assert s.only_compute_if_has_been_stimulated and s.skip_close_to_equilibrium
    s = S.parse_settings(reference_settings(onlyComputeIfHasBeenStimulated=False,
                                            disableComputationWhenStatesAreCloseToEquilibrium=False))
    assert not s.only_compute_if_has_been_stimulated and not s.skip_close_to_equilibrium
    assert s.n_fibers == 2 and s.n_nodes == 42
    np.testing.assert_allclose(s.element_lengths, 0.01)
    np.testing.assert_allclose(s.parameters[:, 0], [0.0, 120.0, 36.0])


def test_compute_state_information_slot_from_settings():
    # the extra slot exists when the diffusion solver has more additional field variables than
    # algebraicsForTransfer (initialization.tpp:572-587)
    cfg = reference_settings()
    assert not S.parse_settings(cfg).compute_state_information
    for inst in cfg["RepeatedCall"]["MultipleInstances"]["instances"][0]["StrangSplitting"]["Term2"][
            "MultipleInstances"]["instances"]:
        inst["ImplicitEuler"]["nAdditionalFieldVariables"] = 1
    assert S.parse_settings(cfg).compute_state_information
    for inst in cfg["RepeatedCall"]["MultipleInstances"]["instances"][0]["StrangSplitting"]["Term1"][
            "MultipleInstances"]["instances"]:
        inst["Heun"]["CellML"]["algebraicsForTransfer"] = [4]
    assert not S.parse_settings(cfg).compute_state_information
