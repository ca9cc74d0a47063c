"""Meshes that mix element types (EMG_ELEM_MIXED: rows of 8 node slots + the
element type, 12 edge slots per element) on the CPU: the oracle's and the
product's numbering against the reference's own code (bit-exact, through the
reference bridge where it is built), the oracle's assembled systems (every
discrete gradient in the kernel of K, a constant-curl field's energy
nu |B0|^2 V: conformity across element types, with the hexahedron's edge
functions at unit circulation), and the rejection of malformed rows and of
the paths that take one element type only."""
import ctypes as C

import numpy as np
import pytest

from emagddm_b200 import _abi, api, mesh
from oracle import oracle as O
from oracle import refbridge as R

LAYOUTS = [("hex_prism", mesh.mixed_hex_prism), ("prism_tet", mesh.mixed_prism_tet),
           ("hex_pyramid_prism", mesh.mixed_hex_pyramid_prism)]


def product_maps(m, gauge=api.GaugeMode.REF, holes=0):
    md = api.EMMeshData(xyz=m.xyz, tets=m.tets, boundary_markers=[
        api.BoundaryMarker(0, "DIRICHLET", "VECTOR_EDGE_ONLY", m.dirichlet, 0.0, "outer")] + [
        api.BoundaryMarker(1 + h, "NEUMANN", "VECTOR_EDGE_ONLY", None, 0.0, f"hole_{h}") for h in range(holes)])
    g = api.GlobalEdgeIDGenerator(md)
    g.generate()
    dm = api.EMDOFManager(md, None, g)
    dm.build()
    dm.applyTreeGauge(gauge)
    return g.getElemLocalToGlobalEdge(), dm.getElemLocalToGlobal()


@pytest.mark.parametrize("name,make", LAYOUTS)
def test_layouts_cover_their_types(name, make):
    m = make(4)
    assert m.elem_type == mesh.ELEM_MIXED
    types = set(np.unique(m.tets[:, 8]))
    assert len(types) >= 2 and types <= {0, 1, 2, 3}
    for t, row in zip(m.tets[:, 8], m.tets):
        assert (row[mesh.NODES_OF_TYPE[t]:8] == -1).all()


@pytest.mark.parametrize("name,make", LAYOUTS)
def test_product_numbering_matches_oracle(name, make):
    m = make(4)
    for holes in (0, 2):
        o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF, n_holes=holes)
        ee, l2g = product_maps(m, holes=holes)
        np.testing.assert_array_equal(ee, o["elem_edge"])
        np.testing.assert_array_equal(l2g, o["l2g"])
        # slots past an element's edges stay -1
        for t, row in zip(m.tets[:, 8], l2g):
            assert (row[mesh.EDGES_OF_TYPE[t]:] == -1).all()


@pytest.mark.skipif(not R.available(), reason="reference bridge not built")
@pytest.mark.parametrize("name,make", LAYOUTS)
def test_numbering_matches_reference_bridge(name, make):
    m = make(4)
    rng = np.random.default_rng(5)
    for d in (m.dirichlet, m.dirichlet[rng.permutation(len(m.dirichlet))[::2]], np.zeros((0, 2), np.int32)):
        for gauge, rg in ((O.GAUGE_REF, True), (O.GAUGE_NONE, False)):
            r = R.dof_build(len(m.xyz), m.tets, d, gauge=rg)
            o = O.dof_build(m.tets, d, gauge=gauge)
            np.testing.assert_array_equal(r["elem_edge"], o["elem_edge"])
            np.testing.assert_array_equal(r["l2g"], o["l2g"])


@pytest.mark.parametrize("name,make", LAYOUTS)
def test_gradients_in_kernel_and_constant_curl_energy(name, make):
    m = mesh.perturbed(make(4), 0.2, seed=3)
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_NONE)
    rp, col, kv, _, _ = O.assemble(m, o["l2g"], o["n_dofs"])
    _, en = O.edge_ids(m.tets)
    phi = np.random.default_rng(0).standard_normal(m.n_nodes)
    phi[np.unique(m.dirichlet)] = 0.0
    g = np.zeros(o["n_dofs"])
    ok = o["edge_dof"] >= 0
    g[o["edge_dof"][ok]] = (phi[en[:, 1]] - phi[en[:, 0]])[ok]
    assert np.abs(O.spmv(rp, col, kv, g)).max() <= 1e-12 * np.abs(kv).max() * np.abs(g).max()
    # constant curl on the unperturbed (affine) mesh, no boundary conditions
    m0 = make(3)
    o = O.dof_build(m0.tets, np.zeros((0, 2), np.int32), gauge=O.GAUGE_NONE)
    rp, col, kv, _, _ = O.assemble(m0, o["l2g"], o["n_dofs"])
    _, en = O.edge_ids(m0.tets)
    B0 = np.array([0.3, -0.2, 0.7])
    x = m0.xyz
    a = np.zeros(o["n_dofs"])
    a[o["edge_dof"]] = np.einsum("ij,ij->i", 0.5 * np.cross(B0, 0.5 * (x[en[:, 0]] + x[en[:, 1]])),
                                 x[en[:, 1]] - x[en[:, 0]])
    assert a @ O.spmv(rp, col, kv, a) == pytest.approx(m0.nu[0] * B0 @ B0, rel=1e-13)


def create(rows, n_nodes):
    h = C.c_void_p()
    rows = np.ascontiguousarray(rows, np.int32)
    rc = _abi.lib().emg_mesh_create_typed(mesh.ELEM_MIXED, n_nodes, None, rows.shape[0], _abi.ptr(rows), None, 0,
                                          None, 0, C.byref(h))
    if rc == 0:
        _abi.lib().emg_mesh_destroy(h)
    return rc


def test_malformed_rows_are_rejected():
    m = mesh.mixed_prism_tet(2)
    assert create(m.tets, m.n_nodes) == 0
    bad = m.tets.copy()
    bad[0, 8] = 7                      # unknown type
    assert create(bad, m.n_nodes) == _abi.EMG_INVALID_INPUT
    bad = m.tets.copy()
    r = int(np.nonzero(bad[:, 8] == 0)[0][0])
    bad[r, 5] = 0                      # a tet row with a node in an unused slot
    assert create(bad, m.n_nodes) == _abi.EMG_INVALID_INPUT


def test_av_map_rejects_mixed_meshes():
    m = mesh.mixed_prism_tet(2)
    rows = np.ascontiguousarray(m.tets, np.int32)
    h = C.c_void_p()
    L = _abi.lib()
    assert L.emg_mesh_create_typed(mesh.ELEM_MIXED, m.n_nodes, None, rows.shape[0], _abi.ptr(rows), None, 0, None, 0,
                                   C.byref(h)) == 0
    try:
        dof_type = np.full(rows.shape[0], 2, np.int32)
        l2g = np.empty(rows.shape[0] * 21, np.int32)
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        assert L.emg_dof_build_av(h, _abi.ptr(dof_type), 0, None, 0, _abi.ptr(l2g), C.byref(a), C.byref(b),
                                  C.byref(c)) == _abi.EMG_INVALID_INPUT
    finally:
        L.emg_mesh_destroy(h)


def test_partitioned_gauge_on_mixed_mesh():
    """The partitioned gauge (FETI-DP's numbering) on a mixed mesh: every
    subdomain's DOFs stay connected and the map is a proper gauge (every free
    edge numbered or in the tree)."""
    from emagddm_b200 import fetidp
    m = mesh.mixed_hex_pyramid_prism(4)
    part = mesh.jittered_partition(m, 2)
    pm = fetidp.partitioned_dofmap(m, part, 8)
    assert pm.l2g.shape == (m.n_tets, 12)
    for t, row in zip(m.tets[:, 8], pm.l2g):
        assert (row[mesh.EDGES_OF_TYPE[t]:] == -1).all()
    assert pm.n_dofs > 0
