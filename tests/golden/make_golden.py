"""Extract the reference's golden vectors for the hot path into cellml_golden.json.

Reads the reference checkout (default /root/reference, or $OPENDIHU_REFERENCE) as TEXT:
  testing/unit_testing/src/1_rank/cellml.cpp  - CellMLTest.HodgkinHuxley{Simd,Vc,OpenMp} and
      CellMLTest.ShortenOpenCOR: the states after 90001 explicit Euler steps of dt=1e-5 (the
      PythonFile output "out_0000009.py" compared at 1e-13 by assertFileMatchesContent);
  testing/unit_testing/input/MU_fibre_distribution_10MUs.txt, MU_firing_times_always.txt -
      summarised (lengths, sums, first entries) to pin the input parsers.
  testing/unit_testing/src/1_rank/laplace_3d.cpp - LaplaceTest.StructuredDeformableMatrixIsCorrect3DStencils:
      the mesh (elements, extent, quadrature) and the element stencil of the expected 3D Laplace stiffness
      matrix, into laplace3d_golden.json (pins the EMG stiffness assembly's values, sign and node order).
The fixtures are committed; nothing at test time reads the reference.
"""
import json
import os
import re
import sys

REF = os.environ.get("OPENDIHU_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from opendihu_b200 import inputs  # noqa: E402


def values_block(src, start, stop):
    blk = src[src.index(start):src.index(stop)]
    vals = [float(v) for v in re.findall(r'\\"values\\": \[([-0-9.e+]+)\]', blk)]
    settings = blk[:blk.index("DihuContext")]
    return vals[3:], settings  # skip the geometry x, y, z


def main():
    src = open(os.path.join(REF, "testing/unit_testing/src/1_rank/cellml.cpp")).read()
    hh, hh_settings = values_block(src, "TEST(CellMLTest, HodgkinHuxleySimd)", "TEST(CellMLTest, HodgkinHuxleyVc)")
    sh, sh_settings = values_block(src, "TEST(CellMLTest, ShortenOpenCOR)", "TEST(CellMLTest, FastFibersVc)")
    assert '"statesInitialValues": [-20, 0.05, 0.6, 0.325]' in hh_settings
    assert '"parametersInitialValues": [400.0]' in hh_settings
    assert '"parametersInitialValues": [1000.0, 1.0]' in sh_settings
    fd = open(os.path.join(REF, "testing/unit_testing/input/MU_fibre_distribution_10MUs.txt")).read()
    ft = open(os.path.join(REF, "testing/unit_testing/input/MU_firing_times_always.txt")).read()
    mus = inputs.parse_fiber_distribution(fd)
    rows = inputs.parse_firing_times(ft)
    out = {
        "source": "testing/unit_testing/src/1_rank/cellml.cpp (CellMLTest.HodgkinHuxleySimd, CellMLTest.ShortenOpenCOR)",
        "explicit_euler": {"dt": 1e-5, "n_steps": 90001, "tolerance": 1e-13},
        "hodgkin_huxley_1952": {"states_initial": [-20, 0.05, 0.6, 0.325],
                                "parameters": {"I_Stim (CONSTANTS[2])": 400.0}, "states_final": hh},
        "shorten_ocallaghan_davidson_soboleva_2007": {
            "states_initial": "model file", "parameters": {"ALGEBRAIC[32]": 1000.0, "CONSTANTS[65]": 1.0},
            "states_final": sh},
        "MU_fibre_distribution_10MUs.txt": {"n": len(mus), "sum": int(sum(mus)), "first": mus[:10],
                                            "last": mus[-10:]},
        "MU_firing_times_always.txt": {"rows": len(rows), "cols": [len(r) for r in rows],
                                       "sum": int(sum(map(sum, rows)))},
    }
    with open(os.path.join(HERE, "cellml_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "cellml_golden.json"))
    laplace_3d()


def laplace_3d():
    name = "TEST(LaplaceTest, StructuredDeformableMatrixIsCorrect3DStencils)"
    src = open(os.path.join(REF, "testing/unit_testing/src/1_rank/laplace_3d.cpp")).read()
    blk = src[src.index(name):src.index("TEST(LaplaceTest, SolverManagerWorks)")]
    n_el = [int(v) for v in re.search(r'"nElements": \[([0-9, ]+)\]', blk).group(1).split(",")]
    ext = [float(v) for v in re.search(r'"physicalExtent": \[([0-9., ]+)\]', blk).group(1).split(",")]
    assert "StructuredDeformableOfDimension<3>" in blk and "Quadrature::Gauss<2>" in blk
    body = blk[blk.index("stencil[2][2][2] = {"):]
    body = body[:body.index("};")]
    nums = re.findall(r"(-?[0-9.]+)/([0-9.]+)", body)
    st = [float(a) / float(b) for a, b in nums]
    assert len(st) == 8
    # the test's element loop: node (x, y, z) numbered z*25 + y*5 + x, entry (i, j) at j*125 + i, the stencil
    # indexed [dy][dx][dz] by the offsets between the two corners of an element
    assert "int node1 = z*25 + y*5 + x+1;" in blk and "stencil[0][1][0]" in blk
    assert "return j*125+i;" in blk
    out = {"source": "testing/unit_testing/src/1_rank/laplace_3d.cpp (" + name[5:-1] + ")",
           "n_elements": n_el, "physical_extent": ext, "quadrature": "Gauss 2",
           "stencil_dy_dx_dz": [[[st[0], st[1]], [st[2], st[3]]], [[st[4], st[5]], [st[6], st[7]]]],
           "node_number": "z*(nx+1)*(ny+1) + y*(nx+1) + x", "tolerance": 1e-14}
    with open(os.path.join(HERE, "laplace3d_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "laplace3d_golden.json"))


if __name__ == "__main__":
    main()
