"""HEX8_EDGE on the CPU: the oracle's hexahedral edge element and numbering
against the reference (golden fixtures from tests/golden/make_golden.py and,
where the reference bridge is built, the reference's own code directly), the
product's host numbering against both, and closed forms of the element.

Parity bars: edge IDs, DOF maps and CSR patterns bit-exact; basis values
exact; curls exact on the 8 edges the reference differentiates correctly and
equal to central differences of the reference's own basis (1e-7) on all 12;
element integrals to 1e-12 of their scale."""
import json
import os

import numpy as np
import pytest

from emagddm_b200 import api, mesh
from oracle import oracle as O
from oracle import refbridge as R

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIX = np.load(os.path.join(GOLD, "reference_hex_fixtures.npz"))
COUNTS = json.load(open(os.path.join(GOLD, "reference_hex_counts.json")))
HEX_EDGES = mesh.HEX_EDGES
# curlHex8Edge (nedelec_element.cpp:618-720) has sign / component errors here
REF_CURL_DEFECTS = (2, 3, 6, 7)


def product_maps(xyz, hexes, dirichlet, holes=0, gauge=api.GaugeMode.REF):
    md = api.EMMeshData(xyz=xyz, tets=hexes, boundary_markers=[
        api.BoundaryMarker(0, "DIRICHLET", "VECTOR_EDGE_ONLY", dirichlet, 0.0, "outer")] + [
        api.BoundaryMarker(1 + h, "NEUMANN", "VECTOR_EDGE_ONLY", None, 0.0, f"hole_{h}") for h in range(holes)])
    g = api.GlobalEdgeIDGenerator(md)
    g.generate()
    dm = api.EMDOFManager(md, None, g)
    dm.build()
    free = dm.getElemLocalToGlobal().copy()
    dm.applyTreeGauge(gauge)
    return g.getElemLocalToGlobalEdge(), free, dm.getElemLocalToGlobal(), dm


@pytest.mark.parametrize("n", [1, 2, 3, 4, 6])
@pytest.mark.parametrize("holes", [0, 2])
def test_hex_counts_match_reference(n, holes):
    xyz, hexes, d = mesh.hex_topology(n)
    o = O.dof_build(hexes, d, gauge=O.GAUGE_REF, n_holes=holes)
    c = COUNTS[f"hex_n{n}_h{holes}"]
    assert (o["n_edges"], o["n_free"], o["n_dofs"]) == (c["n_edges"], c["n_free"], c["n_dofs"])
    assert len(d) == c["n_dirichlet"]


@pytest.mark.parametrize("key", ["hex_n2_h0", "hex_n2_h2", "hex_n3_h0", "hex_n3_h2", "hex_n4_h0", "hex_n4_h2"])
def test_hex_maps_match_reference(key):
    n, holes = int(key[5:key.index("_", 4)]), int(key[-1])
    xyz, hexes, d = mesh.hex_topology(n)
    free = O.dof_build(hexes, d, gauge=O.GAUGE_NONE, n_holes=holes)
    gauge = O.dof_build(hexes, d, gauge=O.GAUGE_REF, n_holes=holes)
    np.testing.assert_array_equal(gauge["elem_edge"], FIX[f"{key}_elem_edge"])
    np.testing.assert_array_equal(free["l2g"], FIX[f"{key}_l2g_free"])
    np.testing.assert_array_equal(gauge["l2g"], FIX[f"{key}_l2g_gauge"])
    # the product's host numbering (emg_mesh_create_typed + emg_dof_build)
    ee, pf, pg, _ = product_maps(xyz, hexes, d, holes)
    np.testing.assert_array_equal(ee, FIX[f"{key}_elem_edge"])
    np.testing.assert_array_equal(pf, FIX[f"{key}_l2g_free"])
    np.testing.assert_array_equal(pg, FIX[f"{key}_l2g_gauge"])


def test_hex_partial_dirichlet_and_pattern_match_reference():
    xyz, hexes, d = mesh.hex_topology(3)
    o = O.dof_build(hexes, d[::3], gauge=O.GAUGE_REF)
    np.testing.assert_array_equal(o["l2g"], FIX["hex_n3_partial_l2g_gauge"])
    _, _, pg, _ = product_maps(xyz, hexes, d[::3])
    np.testing.assert_array_equal(pg, FIX["hex_n3_partial_l2g_gauge"])
    g = O.dof_build(hexes, d, gauge=O.GAUGE_REF)
    rp, col = O.pattern(g["l2g"], g["n_dofs"])
    np.testing.assert_array_equal(rp, FIX["hex_n3_pattern_row_ptr"])
    np.testing.assert_array_equal(col, FIX["hex_n3_pattern_col"])
    assert COUNTS["hex_n3_h0"]["nnz"] == rp[-1]


def test_hex_basis_quadrature_jacobian_fixtures():
    W, Cu = O.hex_basis([0.3, -0.2, 0.5])
    np.testing.assert_array_equal(W, FIX["hex_w_at_0.3_-0.2_0.5"])
    ok = [k for k in range(12) if k not in REF_CURL_DEFECTS]
    np.testing.assert_array_equal(Cu[ok], FIX["hex_curl_at_0.3_-0.2_0.5"][ok])
    for k in REF_CURL_DEFECTS:  # the literal defects stay visible
        assert np.abs(Cu[k] - FIX["hex_curl_at_0.3_-0.2_0.5"][k]).max() > 0.1
    # HEX8 2x2x2 Gauss-Legendre (weights 1, xi outermost); HEX8_EDGE: none
    g = 1 / np.sqrt(3)
    pts = np.array([[(-g, g)[(q >> 2) & 1], (-g, g)[(q >> 1) & 1], (-g, g)[q & 1], 1.0] for q in range(8)])
    np.testing.assert_allclose(FIX["quad_hex8_order8"], pts, rtol=0, atol=1e-15)
    assert FIX["quad_hex8edge_order8"].shape == (0, 4)
    assert np.all(FIX["integrator_k_unit_hex"] == 0.0)  # the reference's literal K_e
    J, det = O.hex_jacobian(FIX["hex_distorted_nodes"], [0.1, 0.2, -0.3])
    np.testing.assert_allclose(J, FIX["hex_distorted_jacobian_at_0.1_0.2_-0.3"], rtol=0, atol=1e-15)
    assert det == pytest.approx(FIX["hex_distorted_det"][0], rel=1e-14)


@pytest.mark.skipif(not R.available(), reason="reference bridge not built")
def test_hex_curls_are_derivatives_of_reference_basis():
    rng = np.random.default_rng(3)
    h = 1e-5
    for x in rng.uniform(-1, 1, (6, 3)):
        W, Cu = O.hex_basis(x)
        Wr, Cr = R.nedelec_hex8(*x)
        np.testing.assert_array_equal(W, Wr)
        # curl by central differences of the reference's evalHex8Edge
        D = np.empty((12, 3, 3))  # D[k, comp, axis]
        for a in range(3):
            e = np.zeros(3)
            e[a] = h
            D[:, :, a] = (R.nedelec_hex8(*(x + e))[0] - R.nedelec_hex8(*(x - e))[0]) / (2 * h)
        curl_fd = np.stack([D[:, 2, 1] - D[:, 1, 2], D[:, 0, 2] - D[:, 2, 0], D[:, 1, 0] - D[:, 0, 1]], axis=1)
        np.testing.assert_allclose(Cu, curl_fd, rtol=0, atol=1e-7)
        ok = [k for k in range(12) if k not in REF_CURL_DEFECTS]
        np.testing.assert_array_equal(Cu[ok], Cr[ok])


@pytest.mark.skipif(not R.available(), reason="reference bridge not built")
@pytest.mark.parametrize("n", [2, 3, 5])
def test_hex_numbering_vs_reference_bridge(n):
    xyz, hexes, d = mesh.hex_topology(n)
    rng = np.random.default_rng(n)
    for dd in (d, d[rng.permutation(len(d))[: len(d) // 2]], np.zeros((0, 2), np.int32)):
        for holes in (0, 1, 3):
            r = R.dof_build(len(xyz), hexes, dd, gauge=True, n_holes=holes)
            o = O.dof_build(hexes, dd, gauge=O.GAUGE_REF, n_holes=holes)
            np.testing.assert_array_equal(r["elem_edge"], o["elem_edge"])
            np.testing.assert_array_equal(r["l2g"], o["l2g"])
            _, _, pg, _ = product_maps(xyz, hexes, dd, holes)
            np.testing.assert_array_equal(pg, r["l2g"])
    r = R.dof_build(len(xyz), hexes, d, gauge=True)
    rp, col, _ = R.pattern(xyz, hexes, r["l2g"])
    rp2, col2 = O.pattern(r["l2g"], int(r["l2g"].max()) + 1)
    np.testing.assert_array_equal(rp, rp2)
    np.testing.assert_array_equal(col, col2)


@pytest.mark.skipif(not R.available(), reason="reference bridge not built")
def test_hex_jacobian_vs_reference_bridge():
    rng = np.random.default_rng(5)
    xyz, hexes, _ = mesh.hex_topology(2)
    for t in range(4):
        X = xyz[hexes[t]] + 0.08 * rng.standard_normal((8, 3))
        for x in rng.uniform(-1, 1, (3, 3)):
            J, det = O.hex_jacobian(X, x)
            Jr, detr = R.hex8_jacobian(X, *x)
            np.testing.assert_allclose(J, Jr, rtol=0, atol=1e-15)
            assert det == pytest.approx(detr, rel=1e-13)


def circulation(u, xa, xb, ng=6):
    g, w = np.polynomial.legendre.leggauss(ng)
    return sum(wi / 2 * np.dot(u(xa + (gi + 1) / 2 * (xb - xa)), xb - xa) for gi, wi in zip(g, w))


def box(scale=(1.0, 2.0, 0.5), shift=(0.3, -0.1, 0.2)):
    xyz, hexes, _ = mesh.hex_topology(1)
    return xyz[hexes[0]] * np.array(scale) + np.array(shift)


def test_hex_element_closed_forms():
    X = box()
    vol = 1.0 * 2.0 * 0.5
    K, M, F = O.element_hex(X, nu=2.0, sigma=3.0, flags=O.FLAG_MASS)
    assert np.abs(K - K.T).max() == 0.0 and np.abs(M - M.T).max() == 0.0
    assert np.linalg.eigvalsh(K).min() > -1e-12 * np.abs(K).max()
    assert np.linalg.eigvalsh(M).min() > 0.0
    # the basis has circulation 4 along its own edge: DOF = circulation / 4
    dofs = lambda u: np.array([circulation(u, X[a], X[b]) for a, b in HEX_EDGES]) / 4.0
    # u = (-y, x, 0) / 2 lies in the space on a box; curl u = e_z
    u = lambda p: np.array([-p[1], p[0], 0.0]) / 2
    a = dofs(u)
    assert a @ K @ a == pytest.approx(2.0 * vol, rel=1e-12)
    # constant field: mass exact under 2x2x2 Gauss, zero curl energy
    a1 = dofs(lambda p: np.array([0.3, -1.0, 0.7]))
    assert a1 @ M @ a1 == pytest.approx(3.0 * vol * (0.09 + 1.0 + 0.49), rel=1e-12)
    assert abs(a1 @ K @ a1) < 1e-12 * np.abs(K).max()
    # source: F . a = int u . J for uniform J inside the element
    src = [mesh.Source(mesh.SRC_BOX, (0.2, 0.5, -1.0), (-9, 9, -9, 9, -9, 9))]
    _, _, F = O.element_hex(X, sources=src)
    assert F @ a1 == pytest.approx(vol * (0.3 * 0.2 - 0.5 + -0.7), rel=1e-12)


def test_hex_gradients_in_kernel_on_distorted_mesh():
    """K G = 0 for every discrete gradient, element by element and assembled
    (the de Rham property the tree-cotree gauge relies on)."""
    m = mesh.perturbed(mesh.hex_small(4), amplitude=0.25, seed=2)
    rng = np.random.default_rng(0)
    for t in range(0, m.n_tets, 7):
        X = m.xyz[m.tets[t]]
        K, _, _ = O.element_hex(X, nu=1.7)
        phi = rng.standard_normal(8)
        a = (phi[HEX_EDGES[:, 1]] - phi[HEX_EDGES[:, 0]]) / 4.0
        assert np.abs(K @ a).max() <= 1e-13 * np.abs(K).max()
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_NONE)
    rp, col, kv, _, _ = O.assemble(m, o["l2g"], o["n_free"])
    # nodal phi vanishing on the boundary -> gradient DOFs on free edges,
    # global orientation low -> high node ID
    phi = rng.standard_normal(m.n_nodes)
    on_b = np.any((m.xyz < 1e-12) | (m.xyz > 1 - 1e-12), axis=1)
    phi[on_b] = 0.0
    ee, en = O.edge_ids(m.tets)
    g = np.zeros(o["n_free"])
    ok = o["edge_dof"] >= 0
    g[o["edge_dof"][ok]] = ((phi[en[:, 1]] - phi[en[:, 0]]) / 4.0)[ok]
    Kg = O.spmv(rp, col, kv, g)
    assert np.abs(Kg).max() <= 1e-12 * np.abs(kv).max() * max(np.abs(g).max(), 1.0)


def test_hex_signs_make_global_orientation():
    hexes = np.array([[5, 1, 9, 3, 0, 7, 2, 8]], np.int32)
    s = O.edge_signs(hexes[0])
    for k, (a, b) in enumerate(HEX_EDGES):
        assert s[k] == (1 if hexes[0][a] < hexes[0][b] else -1)
