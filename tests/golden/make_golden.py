"""Generate the golden fixtures of tests/golden from the reference itself.

Run in a checkout where oracle/_ref/libemg_ref.so has been built from the
reference sources (`make -C oracle -f Makefile.ref`).  Every fixture comes
from the reference's own code path (GlobalEdgeIDGenerator, EMDOFManager,
TreeGauge, EMAssembly + SparseConverter, CGSolver, BiCGSTABSolver,
NedelecElement, GaussQuadrature, MagneticVector3DIntegrator) on the synthetic
Kuhn-split cube meshes of emagddm_b200.mesh:

  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from emagddm_b200 import mesh  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import refbridge as R  # noqa: E402


def main():
    assert R.available(), "build oracle/_ref first (make -C oracle -f Makefile.ref)"
    counts = {}
    arrays = {}
    for n in (1, 2, 3, 4, 6, 8):
        m = mesh.plain_small(n)
        for holes in (0, 2):
            r0 = R.dof_build(m.n_nodes, m.tets, m.dirichlet, gauge=False, n_holes=holes)
            r1 = R.dof_build(m.n_nodes, m.tets, m.dirichlet, gauge=True, n_holes=holes)
            key = f"n{n}_h{holes}"
            counts[key] = dict(n_edges=r1["n_edges"], n_free=r1["n_free"], n_dofs=r1["n_dofs"],
                               n_dirichlet=int(len(m.dirichlet)))
            if n in (2, 3, 4) or (n == 6 and holes == 0):
                arrays[f"{key}_elem_edge"] = r1["elem_edge"].astype(np.int32)
                arrays[f"{key}_l2g_free"] = r0["l2g"].astype(np.int32)
                arrays[f"{key}_l2g_gauge"] = r1["l2g"].astype(np.int32)
    # merged CSR pattern of the gauged system (EMAssembly + to_eigen)
    for n in (3, 4):
        m = mesh.plain_small(n)
        r1 = R.dof_build(m.n_nodes, m.tets, m.dirichlet, gauge=True)
        rp, col, raw = R.pattern(m.xyz, m.tets, r1["l2g"])
        arrays[f"n{n}_pattern_row_ptr"] = rp.astype(np.int64)
        arrays[f"n{n}_pattern_col"] = col.astype(np.int32)
        counts[f"n{n}_h0"]["raw_nnz"] = int(raw)
        counts[f"n{n}_h0"]["nnz"] = int(rp[-1])
    # reference solvers on the restated n=4 system (box source)
    m = mesh.plain_small(4)
    r1 = R.dof_build(m.n_nodes, m.tets, m.dirichlet, gauge=True)
    rp, col, kv, _, rhs = O.assemble(m, r1["l2g"], r1["n_dofs"])
    arrays["solve_n4_row_ptr"] = rp.astype(np.int64)
    arrays["solve_n4_col"] = col.astype(np.int32)
    arrays["solve_n4_val"] = kv
    arrays["solve_n4_rhs"] = rhs
    for kind, name in ((0, "cg"), (1, "bicgstab")):
        for pc in (0, 1):
            x, st, it, res, _, _ = R.krylov(kind, rp, col, kv, rhs, tol=1e-10, max_iter=1000, precond=pc)
            arrays[f"solve_n4_{name}_p{pc}_x"] = x
            counts[f"solve_n4_{name}_p{pc}"] = dict(status=int(st), iterations=int(it), residual=float(res))
    # basis / quadrature / integrator known answers
    w, c = R.nedelec_tet4(0.1, 0.2, 0.3)
    arrays["nedelec_w_at_0.1_0.2_0.3"] = w
    arrays["nedelec_curl"] = c
    arrays["quad_tet4_order4"] = R.quadrature(0, 4)
    arrays["quad_tet4edge_order4"] = R.quadrature(1, 4).reshape(-1, 4)
    X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
    arrays["integrator_k_unit_tet"] = R.integrator_k(X, 1.0)
    np.savez_compressed(os.path.join(HERE, "reference_fixtures.npz"), **arrays)
    with open(os.path.join(HERE, "reference_counts.json"), "w") as f:
        json.dump(counts, f, indent=1, sort_keys=True)
    print("wrote", len(arrays), "arrays and", len(counts), "count records")


if __name__ == "__main__":
    main()
