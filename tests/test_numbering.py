"""Host integer numbering of the product library (C ABI, no GPU needed):
edge IDs, free-DOF map and tree gauge must be bit-exact to the reference
(golden fixtures) and to the oracle."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from emagddm_b200 import _abi, api, mesh
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIX = np.load(os.path.join(GOLD, "reference_fixtures.npz"))
COUNTS = json.load(open(os.path.join(GOLD, "reference_counts.json")))


def product_maps(m, holes=0, mode=api.GaugeMode.REF):
    md = api.EMMeshData.from_cube(m)
    for h in range(holes):
        md.boundary_markers.append(api.BoundaryMarker(1 + h, "NEUMANN", "VECTOR_EDGE_ONLY",
                                                      np.zeros((0, 2), np.int32), 0.0, f"inner_hole_{h}"))
    gen = api.GlobalEdgeIDGenerator(md)
    gen.generate()
    dm = api.EMDOFManager(md, gen.getElemLocalToGlobalEdge(), gen)
    dm.build()
    free = dm.getElemLocalToGlobal().copy()
    nf = dm.getNumFreeDOFs()
    dm.applyTreeGauge(mode)
    return gen, free, nf, dm


@pytest.mark.parametrize("key", ["n2_h0", "n2_h2", "n3_h0", "n3_h2", "n4_h0", "n4_h2", "n6_h0"])
def test_maps_bit_exact_to_reference(key):
    n, holes = int(key[1:key.index("_")]), int(key[-1])
    gen, free, nf, dm = product_maps(mesh.plain_small(n), holes)
    np.testing.assert_array_equal(gen.getElemLocalToGlobalEdge(), FIX[f"{key}_elem_edge"])
    np.testing.assert_array_equal(free, FIX[f"{key}_l2g_free"])
    np.testing.assert_array_equal(dm.getElemLocalToGlobal(), FIX[f"{key}_l2g_gauge"])
    c = COUNTS[key]
    assert (gen.getNumGlobalEdges(), nf, dm.getNumFreeDOFs()) == (c["n_edges"], c["n_free"], c["n_dofs"])


@pytest.mark.parametrize("n,seed", [(5, 1), (7, 2), (12, 3), (16, 4)])
@pytest.mark.parametrize("mode", [api.GaugeMode.REF, api.GaugeMode.BOUNDARY_FIRST])
def test_maps_match_oracle(n, seed, mode):
    m = mesh.random_instance(n, seed)
    gen, free, nf, dm = product_maps(m, 0, mode)
    o = O.dof_build(m.tets, m.dirichlet, gauge=int(mode))
    np.testing.assert_array_equal(gen.getElemLocalToGlobalEdge(), o["elem_edge"])
    np.testing.assert_array_equal(gen.getEdgeNodes(), o["edge_nodes"])
    np.testing.assert_array_equal(dm.getElemLocalToGlobal(), o["l2g"])
    assert dm.getNumFreeDOFs() == o["n_dofs"]


def test_boundary_first_is_a_complete_gauge():
    n = 6
    m = mesh.plain_small(n)
    _, _, nf, dm = product_maps(m, 0, api.GaugeMode.BOUNDARY_FIRST)
    assert dm.getNumFreeDOFs() == nf - (n - 1) ** 3


def test_edge_lookup_and_expand():
    m = mesh.plain_small(3)
    gen, _, _, dm = product_maps(m)
    en = gen.getEdgeNodes()
    for e in (0, 5, len(en) - 1):
        assert gen.getGlobalEdgeID(int(en[e, 1]), int(en[e, 0])) == e
    assert gen.getGlobalEdgeID(0, m.n_nodes - 1) == -1
    red = np.arange(dm.getNumFreeDOFs(), dtype=np.float64) + 1.0
    full = dm.mapReducedSolutionToFull(red)
    ed = dm.getEdgeToDOF()
    assert np.all(full[ed < 0] == 0.0)
    np.testing.assert_array_equal(full[ed >= 0], red[ed[ed >= 0]])


def test_disconnected_mesh_components():
    # two separate cubes: the second component's tree grows from its lowest node
    a = mesh.plain_small(2)
    b = mesh.plain_small(2)
    tets = np.concatenate([a.tets, b.tets + a.n_nodes])
    xyz = np.concatenate([a.xyz, b.xyz + 5.0])
    d = a.dirichlet  # only the first cube is constrained
    md = api.EMMeshData(xyz=xyz, tets=tets, boundary_markers=[api.BoundaryMarker(0, target_ids=d)])
    dm = api.EMDOFManager(md)
    dm.build()
    dm.applyTreeGauge()
    o = O.dof_build(tets, d, gauge=O.GAUGE_REF)
    np.testing.assert_array_equal(dm.getElemLocalToGlobal(), o["l2g"])


def test_invalid_inputs_are_rejected():
    L = _abi.lib()
    h = C.c_void_p()
    tets = np.array([[0, 1, 2, 9]], np.int32)
    xyz = np.zeros((4, 3))
    rc = L.emg_mesh_create(4, _abi.ptr(xyz), 1, _abi.ptr(tets), None, 0, None, 0, C.byref(h))
    assert rc == _abi.EMG_INVALID_INPUT
    assert b"out of range" in L.emg_last_error()
    rc = L.emg_mesh_create(0, None, 0, None, None, 0, None, 0, C.byref(h))
    assert rc == _abi.EMG_INVALID_INPUT
    tets = np.array([[0, 1, 2, 3]], np.int32)
    assert L.emg_mesh_create(4, _abi.ptr(xyz), 1, _abi.ptr(tets), None, 0, None, 0, C.byref(h)) == 0
    dm = C.c_void_p()
    assert L.emg_dof_build(h, 7, C.byref(dm)) == _abi.EMG_INVALID_INPUT
    L.emg_mesh_destroy(h)
