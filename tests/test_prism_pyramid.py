"""PRISM6_EDGE and PYRAMID5_EDGE on the CPU: the oracle's reference elements
(unit circulations, gradients of the nodal functions in the edge span), the
oracle's and the product's numbering against the reference's own code (edge
IDs and DOF maps bit-exact, through the reference bridge where it is built),
and two size-independent properties of the oracle's assembled systems: every
discrete gradient lies in the kernel of K, and a field of constant curl B0
has energy nu |B0|^2 V.

The reference assembles these elements with no quadrature points
(getPoints(PRISM6_EDGE / PYRAMID5_EDGE) returns none), so its literal
element matrices are zero; the oracle's formulas are the intended ones,
checked here by the properties above."""
import numpy as np
import pytest

from emagddm_b200 import api, mesh
from oracle import oracle as O
from oracle import refbridge as R

TYPES = [(O.ELEM_PRISM6_EDGE, mesh.prism_small, mesh.prism_scale),
         (O.ELEM_PYRAMID5_EDGE, mesh.pyramid_small, mesh.pyramid_scale)]


@pytest.mark.parametrize("et", [O.ELEM_PRISM6_EDGE, O.ELEM_PYRAMID5_EDGE])
def test_basis_has_unit_circulations(et):
    E = O.edges_per_elem(et)
    C = np.array([[O.shape_circulation(et, k, e) for e in range(E)] for k in range(E)])
    np.testing.assert_allclose(C, np.eye(E), atol=1e-12)


@pytest.mark.parametrize("et", [O.ELEM_PRISM6_EDGE, O.ELEM_PYRAMID5_EDGE])
def test_nodal_gradients_lie_in_the_edge_span(et):
    rng = np.random.default_rng(et)
    for _ in range(20):
        x = rng.uniform([0.0, 0.0, -1.0], [0.5, 0.5, 1.0]) if et == O.ELEM_PRISM6_EDGE else \
            rng.uniform([-1.0, -1.0, 0.0], [1.0, 1.0, 0.95])
        assert O.shape_grad_residual(et, x) <= 1e-14


def product_maps(m, gauge=api.GaugeMode.REF):
    md = api.EMMeshData(xyz=m.xyz, tets=m.tets, boundary_markers=[
        api.BoundaryMarker(0, "DIRICHLET", "VECTOR_EDGE_ONLY", m.dirichlet, 0.0, "outer")])
    g = api.GlobalEdgeIDGenerator(md)
    g.generate()
    dm = api.EMDOFManager(md, None, g)
    dm.build()
    dm.applyTreeGauge(gauge)
    return g.getElemLocalToGlobalEdge(), dm.getElemLocalToGlobal()


@pytest.mark.parametrize("et,small,scale", TYPES)
def test_product_numbering_matches_oracle(et, small, scale):
    for m in (small(3), mesh.perturbed(scale(4), 0.2, seed=1)):
        assert m.elem_type == et
        o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
        ee, l2g = product_maps(m)
        np.testing.assert_array_equal(ee, o["elem_edge"])
        np.testing.assert_array_equal(l2g, o["l2g"])


@pytest.mark.skipif(not R.available(), reason="reference bridge not built")
@pytest.mark.parametrize("et,small,scale", TYPES)
def test_numbering_matches_reference_bridge(et, small, scale):
    for m in (small(3), scale(5)):
        rng = np.random.default_rng(3)
        for d in (m.dirichlet, m.dirichlet[rng.permutation(len(m.dirichlet))[: len(m.dirichlet) // 2]]):
            for gauge, rg in ((O.GAUGE_REF, True), (O.GAUGE_NONE, False)):
                r = R.dof_build(len(m.xyz), m.tets, d, gauge=rg)
                o = O.dof_build(m.tets, d, gauge=gauge)
                np.testing.assert_array_equal(r["elem_edge"], o["elem_edge"])
                np.testing.assert_array_equal(r["l2g"], o["l2g"])


def gradient_dofs(m, o, phi):
    """Edge DOFs of grad(phi) (global orientation low -> high node)."""
    _, en = O.edge_ids(m.tets)
    g = np.zeros(o["n_dofs"])
    ok = o["edge_dof"] >= 0
    g[o["edge_dof"][ok]] = (phi[en[:, 1]] - phi[en[:, 0]])[ok]
    return g


@pytest.mark.parametrize("et,small,scale", TYPES)
def test_gradients_in_kernel_of_oracle_matrix(et, small, scale):
    m = mesh.perturbed(scale(4), 0.25, seed=2)
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_NONE)
    rp, col, kv, _, _ = O.assemble(m, o["l2g"], o["n_dofs"])
    phi = np.random.default_rng(0).standard_normal(m.n_nodes)
    phi[np.unique(m.dirichlet)] = 0.0
    g = gradient_dofs(m, o, phi)
    assert np.abs(O.spmv(rp, col, kv, g)).max() <= 1e-12 * np.abs(kv).max() * np.abs(g).max()


@pytest.mark.parametrize("et,small,scale", TYPES)
def test_constant_curl_energy(et, small, scale):
    """A = B0 x x / 2 is in the span (its DOFs are its edge circulations):
    a^T K a = nu |B0|^2 V, on affine elements to rounding."""
    m = small(3)
    o = O.dof_build(m.tets, np.zeros((0, 2), np.int32), gauge=O.GAUGE_NONE)
    rp, col, kv, _, _ = O.assemble(m, o["l2g"], o["n_dofs"])
    B0 = np.array([0.3, -0.2, 0.7])
    _, en = O.edge_ids(m.tets)
    x = m.xyz
    mid = 0.5 * (x[en[:, 0]] + x[en[:, 1]])
    a = np.zeros(o["n_dofs"])
    a[o["edge_dof"]] = np.einsum("ij,ij->i", 0.5 * np.cross(B0, mid), x[en[:, 1]] - x[en[:, 0]])
    assert a @ O.spmv(rp, col, kv, a) == pytest.approx(m.nu[0] * B0 @ B0, rel=1e-13)
