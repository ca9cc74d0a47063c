"""Gmsh ASCII input (emg_mesh_read_gmsh, formats 2.2 and 4.1): a mesh written
by mesh.write_gmsh reads back to the same arrays, the Dirichlet edges of the
boundary physical group equal the cube's boundary-face edges, and the numbering
of the read mesh equals the oracle's."""
import numpy as np
import pytest

from emagddm_b200 import _abi, mesh
from oracle import oracle as O


def edge_set(pairs):
    p = np.sort(np.asarray(pairs, np.int64), axis=1)
    return set(map(tuple, np.unique(p, axis=0)))


@pytest.mark.parametrize("version", ["2.2", "4.1"])
@pytest.mark.parametrize("by_tag", [True, False])
def test_gmsh_round_trip(tmp_path, version, by_tag):
    m = mesh.perturbed(mesh.plain_scale(5), 0.2, seed=3)
    path = str(tmp_path / f"cube_{version}.msh")
    mesh.write_gmsh(m, path, version=version)
    r = mesh.read_gmsh(path, dirichlet_tags=[100] if by_tag else None)
    # 4.1 stores the tetrahedra in one block per volume entity: file order is
    # grouped by material (stable), and the reader keeps file order
    order = np.arange(m.n_tets) if version == "2.2" else np.argsort(m.material, kind="stable")
    m = mesh.CubeMesh(**{**m.__dict__, "tets": m.tets[order], "material": m.material[order]})
    np.testing.assert_array_equal(r.tets, m.tets)
    np.testing.assert_array_equal(r.material, m.material)
    np.testing.assert_allclose(r.xyz, m.xyz, rtol=0, atol=0)
    np.testing.assert_array_equal(r.material_tags, [1, 2])
    assert edge_set(r.dirichlet) == edge_set(m.dirichlet)
    a = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
    b = O.dof_build(r.tets, r.dirichlet, gauge=O.GAUGE_REF)
    np.testing.assert_array_equal(a["l2g"], b["l2g"])


@pytest.mark.parametrize("version", ["2.2", "4.1"])
@pytest.mark.parametrize("by_tag", [True, False])
def test_gmsh_hex_round_trip(tmp_path, version, by_tag):
    """HEX8 volumes (type 5) with quadrangle boundary faces (type 3): same
    arrays back, Dirichlet edges = the cube's boundary-face edges (no face
    diagonals), the same numbering."""
    m = mesh.perturbed(mesh.hex_scale(4), 0.2, seed=5)
    path = str(tmp_path / f"hex_{version}.msh")
    mesh.write_gmsh(m, path, version=version)
    r = mesh.read_gmsh(path, dirichlet_tags=[100] if by_tag else None)
    order = np.arange(m.n_tets) if version == "2.2" else np.argsort(m.material, kind="stable")
    m = mesh.CubeMesh(**{**m.__dict__, "tets": m.tets[order], "material": m.material[order]})
    assert r.tets.shape[1] == 8
    np.testing.assert_array_equal(r.tets, m.tets)
    np.testing.assert_array_equal(r.material, m.material)
    np.testing.assert_allclose(r.xyz, m.xyz, rtol=0, atol=0)
    assert edge_set(r.dirichlet) == edge_set(m.dirichlet)
    a = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
    b = O.dof_build(r.tets, r.dirichlet, gauge=O.GAUGE_REF)
    np.testing.assert_array_equal(a["l2g"], b["l2g"])


def test_gmsh_mixed_and_unsupported_volumes(tmp_path):
    head = "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n12\n" + "".join(
        f"{i + 1} {i % 2} {(i // 2) % 2} {i // 4}\n" for i in range(12)) + "$EndNodes\n$Elements\n"
    mixed = tmp_path / "mixed.msh"
    mixed.write_text(head + "2\n1 4 2 1 1 1 2 3 5\n2 5 2 1 1 1 2 4 3 5 6 8 7\n$EndElements\n")
    with pytest.raises(RuntimeError, match="tetrahedra and hexahedra"):
        mesh.read_gmsh(str(mixed))
    prism = tmp_path / "prism.msh"
    prism.write_text(head + "1\n1 6 2 1 1 1 2 3 5 6 7\n$EndElements\n")
    with pytest.raises(RuntimeError, match="prism"):
        mesh.read_gmsh(str(prism))
    hex20 = tmp_path / "hex20.msh"
    hex20.write_text(head + "1\n1 17 2 1 1 " + " ".join(str(1 + i % 12) for i in range(20)) + "\n$EndElements\n")
    with pytest.raises(RuntimeError, match="higher-order hexahedra"):
        mesh.read_gmsh(str(hex20))


def test_gmsh_errors(tmp_path):
    bad = tmp_path / "bad.msh"
    bad.write_text("$MeshFormat\n2.2 1 8\n$EndMeshFormat\n")
    with pytest.raises(RuntimeError, match="binary"):
        mesh.read_gmsh(str(bad))
    with pytest.raises(RuntimeError, match="cannot open"):
        mesh.read_gmsh(str(tmp_path / "missing.msh"))
    q = tmp_path / "quad.msh"
    q.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n10\n" +
                 "".join(f"{i + 1} {i} 0 0\n" for i in range(10)) +
                 "$EndNodes\n$Elements\n1\n1 11 2 1 1 1 2 3 4 5 6 7 8 9 10\n$EndElements\n")
    with pytest.raises(RuntimeError, match="higher-order"):
        mesh.read_gmsh(str(q))


@pytest.mark.gpu
@pytest.mark.parametrize("version", ["2.2", "4.1"])
@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_gmsh_mesh_through_the_gpu_path(tmp_path, version, kind):
    """A perturbed (non-structured geometry) mesh read from Gmsh: GPU assembly
    to 1e-12 of the oracle, CG and the direct backend to 1e-8 of the oracle's solve."""
    from emagddm_b200 import fetidp
    from tests.helpers import System, oracle_system, solve
    src = mesh.perturbed(mesh.plain_scale(8) if kind == "tet" else mesh.hex_scale(8), 0.25, seed=4)
    path = str(tmp_path / "m.msh")
    mesh.write_gmsh(src, path, version=version)
    m = mesh.read_gmsh(path, dirichlet_tags=[100], nu=src.nu, sigma=src.sigma, sources=src.sources)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    s = System(m, l2g)
    rp, col, kv, _, rhs = s.export()
    orp, ocol, okv, _, orhs = oracle_system(m, l2g)
    np.testing.assert_array_equal(col, ocol)
    assert np.abs(kv - okv).max() <= 1e-12 * np.abs(okv).max()
    assert np.abs(rhs - orhs).max() <= 1e-12 * np.abs(orhs).max()
    xo, st, it, _ = O.pcg(orp, ocol, okv, orhs, tol=1e-12, max_iter=20000, precond=1)
    x, out = solve(s.matrix(0), orhs, "cg", tol=1e-12, max_iter=20000)
    assert out.status == 0 and np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
    ds = fetidp.DirectSolver(m)
    assert ds.factor() == 0
    xd, rc, o2 = ds.solve(tol=1e-12)
    assert rc == 0 and np.linalg.norm(xd - xo) <= 1e-8 * np.linalg.norm(xo)
