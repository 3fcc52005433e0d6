"""Writes the golden fixtures of tests/golden/ (run from the repository root:
`python tests/golden/make_golden.py`).

Two kinds of entries:

* known answers restated from the reference's own tests (the constant, the
  inputs and the reference file:line they come from); the reference itself is
  Fortran and cannot be built here, so these constants are what pins the oracle;
* oracle regression vectors for small cases (element stiffness of a distorted
  hex, a J2 history, a small assembled matrix), each cross-checked against the
  independent numpy restatement before it is written.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import np_oracle as N  # noqa: E402
from oracle import oracle as O  # noqa: E402


def known_answers():
    return {
        "umat_elastic_uniaxial_strain": {
            "source": "ufc_core/Testing/test_defn_invoke_umat.f90:20,43",
            "props": [210000.0, 0.3], "dstrain": [1e-3, 0, 0, 0, 0, 0],
            "sigma11": 282.69230769230769, "reference_tol": 1e-5},
        "c3d8_unit_cube_uniaxial": {
            "source": "tests/ufc_core/test_c3d8_uniaxial.f90:1-18,55-57",
            "E": 200e9, "nu": 0.3, "sigma": 100e6, "u_x_face": 5e-4, "u_y_face": -1.5e-4,
            "reference_tol_rel": 1e-2},
        "j2_uniaxial_history": {
            "source": "tests/integration/E2E_C2_02_Uniaxial_J2Plastic.f90:38-41,77-80,108-113,129-202",
            "props": [200000.0, 0.3, 250.0, 1000.0], "eps11": [0.001, 0.002, 0.003, 0.005],
            "lateral": "eps22 = eps33 = -nu * eps11", "elastic_tol_pct": 0.1, "yield_tol_pct": 1.0},
        "perfect_plasticity": {
            "source": "tests/HARNESS_Mat_Plastic_VonMises.f90",
            "props": [200000.0, 0.3, 250.0, 0.0], "q_tol": 1e-10},
        "fd_tangent": {"source": "tests/integration/test_elem_mat_ip_loop.f90:16", "rel_tol": 1e-4},
        "assembly_symmetry": {"source": "tests/integration/test_assembly_chain.f90:37-40", "rel_tol": 1e-14},
        "patch_rigid_body": {"source": "tests/HARNESS_Elem_C3D8_PatchTest.f90", "tol": 1e-6},
    }


def distorted_hex():
    rng = np.random.default_rng(11)
    X = np.array(N.SIGNS * 0.5 + 0.5)
    X += 0.08 * rng.standard_normal(X.shape)
    return X


def regression():
    out = {}
    X = distorted_hex()
    D = N.iso_D(210e3, 0.3)
    K_c = O.c3d8_ke(X, D)
    K_n = N.ke(X, D)
    assert np.abs(K_c - K_n).max() <= 1e-12 * np.abs(K_n).max()
    out["ke_distorted_hex"] = {"X": X.tolist(), "E": 210e3, "nu": 0.3, "Ke": K_c.tolist()}
    props = [200000.0, 0.3, 250.0, 1000.0]
    sig, ep, epl = np.zeros(6), 0.0, np.zeros(6)
    prev = np.zeros(6)
    hist = []
    steps = [np.array([1e-3, -3e-4, -3e-4, 0, 0, 0]), np.array([3e-3, -1e-3, -8e-4, 1e-3, 0, 0]),
             np.array([4e-3, -1e-3, -1e-3, 2e-3, -1e-3, 5e-4]), np.array([2e-3, 0, 0, 0, 0, 0])]
    for tot in steps:
        s, e2, l2, Dep, y = O.j2_update(props, tot - prev, sig, ep, epl)
        s_n, e_n = N.j2_tensor(props, tot - prev, sig, ep)
        assert np.abs(s - s_n).max() <= 1e-9 * max(1.0, np.abs(s).max()) and abs(e2 - e_n) <= 1e-14
        hist.append({"strain": tot.tolist(), "sigma": s.tolist(), "epeq": e2, "eps_p": l2.tolist(),
                     "ddsdde": Dep.tolist(), "yielded": y})
        sig, ep, epl, prev = s, e2, l2, tot
    out["j2_mixed_history"] = {"props": props, "steps": hist}
    import __graft_entry__

    mesh = __graft_entry__.load_package().mesh
    p_small = mesh.cantilever(3, 2, 2, 3.0, 2.0, 2.0, E=np.linspace(1e3, 5e3, 12))
    m = O.Model(p_small)
    K = m.assemble()
    u, info = m.solve_linear(rtol=1e-14)
    out["cantilever_3x2x2"] = {"row_ptr": m.row_ptr.tolist(), "col": m.col.tolist(), "val": K.val.tolist(),
                               "u": u.tolist(), "f": p_small.f.tolist(), "fixed": p_small.fixed.tolist()}
    return out


def main():
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known_answers(), f, indent=1)
    with open(os.path.join(HERE, "oracle_regression.json"), "w") as f:
        json.dump(regression(), f)
    print("wrote", HERE)


if __name__ == "__main__":
    main()
