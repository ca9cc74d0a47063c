"""The C++ adapters (include/emagddm_b200.hpp) driven by a C++ program that
calls them the way a reference caller would (tests/cpp/solve_cube.cpp)."""
import os
import subprocess

import numpy as np
import pytest

from emagddm_b200 import mesh
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cpp", "solve_cube")


def run(*args):
    if not os.path.exists(EXE):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "emagddm_b200", "csrc"), "demo"])
    out = subprocess.run([EXE, *map(str, args)], capture_output=True, text=True, timeout=600)
    kv = dict(t.split("=", 1) for t in out.stdout.split() if "=" in t)
    return out.returncode, kv


@pytest.mark.parametrize("n", [2, 4, 7])
def test_cpp_numbering_matches_oracle(n):
    rc, kv = run(n, "--numbering-only")
    assert rc == 0
    m = mesh.plain_small(n)
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
    assert int(kv["edges"]) == o["n_edges"]
    assert int(kv["free"]) == o["n_free"]
    assert int(kv["dofs"]) == o["n_dofs"]
    assert int(kv["l2g_sum"]) == int(o["l2g"].astype(np.int64).sum())


@pytest.mark.gpu
def test_cpp_chain_solution_matches_oracle(tmp_path):
    n = 6
    xfile = tmp_path / "x.bin"
    rc, kv = run(n, "--x", xfile)
    assert rc == 0, kv
    assert kv["status"] == "0" and kv["solver"] == "CGSolver_Jacobi"
    m = mesh.plain_small(n)
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
    rp, col, kv_, _, rhs = O.assemble(m, o["l2g"], o["n_dofs"])
    xo, st, it, res = O.pcg(rp, col, kv_, rhs, tol=1e-10, max_iter=10000, precond=1)
    x = np.fromfile(xfile, dtype=np.float64)
    assert abs(int(kv["iterations"]) - it) <= max(3, 0.15 * it)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)


@pytest.mark.gpu
def test_cpp_direct_backend_matches_oracle(tmp_path):
    n = 6
    xfile = tmp_path / "xd.bin"
    rc, kv = run(n, "--direct", "--x", xfile)
    assert rc == 0, kv
    assert kv["status"] == "0" and kv["solver"] == "GpuDirectBackend"
    assert float(kv["residual"]) <= 1e-12
    m = mesh.plain_small(n)
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
    rp, col, kv_, _, rhs = O.assemble(m, o["l2g"], o["n_dofs"])
    xo, st, it, res = O.pcg(rp, col, kv_, rhs, tol=1e-12, max_iter=10000, precond=1)
    x = np.fromfile(xfile, dtype=np.float64)
    assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)


@pytest.mark.parametrize("n,hexes", [(3, False), (4, True)])
def test_cpp_dof_types_match_oracle(n, hexes):
    """EMDOFManager::buildWithDofTypes (per-element SCALAR_ONLY /
    VECTOR_EDGE_ONLY / MIXED_AV) from C++ against the oracle."""
    rc, kv = run(n, "--numbering-only", "--av", *(["--hex"] if hexes else []))
    assert rc == 0
    if hexes:
        xyz, el, d = mesh.hex_topology(n)
    else:
        m = mesh.plain_small(n)
        xyz, el, d = m.xyz, m.tets, m.dirichlet
    t = (np.arange(el.shape[0]) % 3).astype(np.int32)
    bnd = np.where(np.any((xyz < 1e-12) | (xyz > 1 - 1e-12), axis=1))[0].astype(np.int32)
    o = O.dof_build_av(el, t, d, bnd, gauge=O.GAUGE_REF, n_nodes=len(xyz))
    rows = o["l2g"]
    assert int(kv["av_dofs"]) == o["n_dofs"] and int(kv["av_scalar"]) == o["n_scalar_free"]
    assert int(kv["av_sum"]) == int(rows[rows != -2].astype(np.int64).sum())
    assert int(kv["av_len"]) == int((rows != -2).sum())


@pytest.mark.parametrize("n", [2, 3, 5])
def test_cpp_hex_numbering_matches_oracle(n):
    rc, kv = run(n, "--numbering-only", "--hex")
    assert rc == 0
    xyz, hexes, d = mesh.hex_topology(n)
    o = O.dof_build(hexes, d, gauge=O.GAUGE_REF)
    assert int(kv["edges"]) == o["n_edges"]
    assert int(kv["free"]) == o["n_free"]
    assert int(kv["dofs"]) == o["n_dofs"]
    assert int(kv["l2g_sum"]) == int(o["l2g"].astype(np.int64).sum())


@pytest.mark.gpu
@pytest.mark.parametrize("direct", [False, True])
def test_cpp_hex_chain_matches_oracle(tmp_path, direct):
    """HEX8_EDGE through the C++ adapters on a non-affine (wiggled) grid."""
    n = 6
    xfile, gfile = tmp_path / "x.bin", tmp_path / "xyz.bin"
    args = [n, "--hex", "--wiggle", "--x", xfile, "--xyz", gfile] + (["--direct"] if direct else [])
    rc, kv = run(*args)
    assert rc == 0, kv
    _, hexes, d = mesh.hex_topology(n)
    xyz = np.fromfile(gfile, dtype=np.float64).reshape(-1, 3)
    m = mesh.CubeMesh(n=n, xyz=xyz, tets=hexes, material=np.zeros(len(hexes), np.int32), dirichlet=d,
                      nu=np.array([1.0]), sigma=np.array([0.0]), sources=mesh.plain_small(n).sources)
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
    rp, col, kv_, _, rhs = O.assemble(m, o["l2g"], o["n_dofs"])
    assert np.abs(rhs).max() > 1e-6
    xo, st, it, res = O.pcg(rp, col, kv_, rhs, tol=1e-12, max_iter=20000, precond=1)
    x = np.fromfile(xfile, dtype=np.float64)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
