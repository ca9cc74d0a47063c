"""Generate the golden fixtures of tests/golden from the reference itself.

Run in a checkout where oracle/_ref/libemg_ref.so has been built from the
reference sources (`make -C oracle -f Makefile.ref`).  Every fixture comes
from the reference's own code path (GlobalEdgeIDGenerator, EMDOFManager,
TreeGauge, EMAssembly + SparseConverter, CGSolver, BiCGSTABSolver,
NedelecElement, GaussQuadrature, MagneticVector3DIntegrator) on the synthetic
Kuhn-split cube meshes of emagddm_b200.mesh, the HEX8_EDGE fixtures on the
hex grids of the same module, and the per-element DOF-type (MIXED_AV)
fixtures on both:

  python tests/golden/make_golden.py [--hex-only | --av-only | --ilu0-only]
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


def hex_fixtures():
    """HEX8_EDGE fixtures (reference_hex_fixtures.npz / reference_hex_counts.json)
    on the n^3 hex grids of emagddm_b200.mesh.hex_topology."""
    counts = {}
    arrays = {}
    for n in (1, 2, 3, 4, 6):
        xyz, hexes, d = mesh.hex_topology(n)
        for holes in (0, 2):
            r0 = R.dof_build(len(xyz), hexes, d, gauge=False, n_holes=holes)
            r1 = R.dof_build(len(xyz), hexes, d, gauge=True, n_holes=holes)
            key = f"hex_n{n}_h{holes}"
            counts[key] = dict(n_edges=r1["n_edges"], n_free=r1["n_free"], n_dofs=r1["n_dofs"],
                               n_dirichlet=int(len(d)))
            if n in (2, 3, 4):
                arrays[f"{key}_elem_edge"] = r1["elem_edge"].astype(np.int32)
                arrays[f"{key}_l2g_free"] = r0["l2g"].astype(np.int32)
                arrays[f"{key}_l2g_gauge"] = r1["l2g"].astype(np.int32)
    # every third Dirichlet pair only (a partly clamped boundary)
    xyz, hexes, d = mesh.hex_topology(3)
    r1 = R.dof_build(len(xyz), hexes, d[::3], gauge=True)
    arrays["hex_n3_partial_l2g_gauge"] = r1["l2g"].astype(np.int32)
    counts["hex_n3_partial"] = dict(n_edges=r1["n_edges"], n_free=r1["n_free"], n_dofs=r1["n_dofs"])
    # merged CSR pattern of the gauged n=3 system
    r1 = R.dof_build(len(xyz), hexes, d, gauge=True)
    rp, col, raw = R.pattern(xyz, hexes, r1["l2g"])
    arrays["hex_n3_pattern_row_ptr"] = rp.astype(np.int64)
    arrays["hex_n3_pattern_col"] = col.astype(np.int32)
    counts["hex_n3_h0"]["raw_nnz"] = int(raw)
    counts["hex_n3_h0"]["nnz"] = int(rp[-1])
    # basis, quadrature, Jacobian, integrator known answers
    w, c = R.nedelec_hex8(0.3, -0.2, 0.5)
    arrays["hex_w_at_0.3_-0.2_0.5"] = w
    arrays["hex_curl_at_0.3_-0.2_0.5"] = c
    arrays["quad_hex8_order8"] = R.quadrature_hex(0, 8)
    arrays["quad_hex8edge_order8"] = R.quadrature_hex(1, 8).reshape(-1, 4)
    X = np.array([[0, 0, 0], [1, 0.1, 0], [1.2, 1, 0.1], [0, 0.9, 0], [0.1, 0, 1], [1, 0, 1.1],
                  [1, 1.1, 1], [0, 1, 0.9]])
    J, det = R.hex8_jacobian(X, 0.1, 0.2, -0.3)
    arrays["hex_distorted_nodes"] = X
    arrays["hex_distorted_jacobian_at_0.1_0.2_-0.3"] = J
    arrays["hex_distorted_det"] = np.array([det])
    arrays["integrator_k_unit_hex"] = R.integrator_k_hex(mesh.hex_topology(1)[0], 1.0)
    np.savez_compressed(os.path.join(HERE, "reference_hex_fixtures.npz"), **arrays)
    with open(os.path.join(HERE, "reference_hex_counts.json"), "w") as f:
        json.dump(counts, f, indent=1, sort_keys=True)
    print("wrote", len(arrays), "hex arrays and", len(counts), "hex count records")


def av_patterns(T):
    """Element::dof_type patterns of the per-element DOF-type fixtures
    (0 SCALAR_ONLY, 1 VECTOR_EDGE_ONLY, 2 MIXED_AV)."""
    half = np.arange(T) < T // 2
    return {"all_av": np.full(T, 2, np.int32),
            "cycle": (np.arange(T) % 3).astype(np.int32),
            "av_vector": np.where(half, 2, 1).astype(np.int32),
            "av_scalar": np.where(half, 2, 0).astype(np.int32)}


def av_meshes():
    m = mesh.plain_small(3)
    yield "tet3", m.xyz, m.tets, m.dirichlet
    xyz, hexes, d = mesh.hex_topology(3)
    yield "hex3", xyz, hexes, d


def av_fixtures():
    """Per-element DOF types (reference_av_fixtures.npz / reference_av_counts.json):
    EMDOFManager with SCALAR_ONLY / VECTOR_EDGE_ONLY / MIXED_AV elements and a
    scalar DIRICHLET marker on every second boundary node."""
    counts = {}
    arrays = {}
    for name, xyz, el, d in av_meshes():
        bnd = np.unique(np.asarray(d).ravel()).astype(np.int32)[::2]
        for pat, dt in av_patterns(el.shape[0]).items():
            for holes in (0, 2):
                for gauge in (False, True):
                    r = R.dof_build_av(len(xyz), el, dt, d, bnd, gauge=gauge, n_holes=holes)
                    key = f"{name}_{pat}_h{holes}_{'gauge' if gauge else 'free'}"
                    arrays[key] = r["l2g"].astype(np.int32)
                    counts[key] = dict(n_free=r["n_free"], n_dofs=r["n_dofs"])
    np.savez_compressed(os.path.join(HERE, "reference_av_fixtures.npz"), **arrays)
    with open(os.path.join(HERE, "reference_av_counts.json"), "w") as f:
        json.dump(counts, f, indent=1, sort_keys=True)
    print("wrote", len(arrays), "per-element DOF-type arrays")


def ilu0_fixtures():
    """The reference's CGSolver / BiCGSTABSolver with PreconditionerType::ILU0
    (Eigen IncompleteLUT inside) on the restated n=4 box-source system and the
    n=6 iron-block / coil system (reference_ilu0_fixtures.npz /
    reference_ilu0_counts.json)."""
    arrays, counts = {}, {}
    for tag, m in (("n4", mesh.plain_small(4)), ("s6", mesh.plain_scale(6))):
        r1 = R.dof_build(m.n_nodes, m.tets, m.dirichlet, gauge=True)
        rp, col, kv, _, rhs = O.assemble(m, r1["l2g"], r1["n_dofs"])
        arrays[f"{tag}_row_ptr"] = rp.astype(np.int64)
        arrays[f"{tag}_col"] = col.astype(np.int32)
        arrays[f"{tag}_val"] = kv
        arrays[f"{tag}_rhs"] = rhs
        for kind, name in ((0, "cg"), (1, "bicgstab")):
            x, st, it, res, _, _ = R.krylov(kind, rp, col, kv, rhs, tol=1e-10, max_iter=1000, precond=2)
            arrays[f"{tag}_{name}_ilu0_x"] = x
            counts[f"{tag}_{name}_ilu0"] = dict(status=int(st), iterations=int(it), residual=float(res))
    np.savez_compressed(os.path.join(HERE, "reference_ilu0_fixtures.npz"), **arrays)
    with open(os.path.join(HERE, "reference_ilu0_counts.json"), "w") as f:
        json.dump(counts, f, indent=1, sort_keys=True)
    print("wrote", len(arrays), "ILU0 arrays:", counts)


def main():
    assert R.available(), "build oracle/_ref first (make -C oracle -f Makefile.ref)"
    R.lib().refb_quiet(1)
    if "--ilu0-only" in sys.argv:
        ilu0_fixtures()
        return
    if "--hex-only" in sys.argv:
        hex_fixtures()
        return
    if "--av-only" in sys.argv:
        av_fixtures()
        return
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
    hex_fixtures()
    av_fixtures()
    ilu0_fixtures()


if __name__ == "__main__":
    main()
