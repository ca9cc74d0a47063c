"""Per-element DOF types (SCALAR_ONLY / VECTOR_EDGE_ONLY / MIXED_AV) in the
host numbering of the product library (C ABI, no GPU needed): maps
bit-exact to the reference's EMDOFManager (golden fixtures made by
tests/golden/make_golden.py from the reference itself) and to the oracle."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from emagddm_b200 import _abi, api, mesh
from oracle import oracle as O
from tests.golden.make_golden import av_meshes, av_patterns

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIX = np.load(os.path.join(GOLD, "reference_av_fixtures.npz"))
COUNTS = json.load(open(os.path.join(GOLD, "reference_av_counts.json")))
MESHES = {name: (xyz, el, d) for name, xyz, el, d in av_meshes()}


def mesh_data(xyz, el, d, dof_type, scalar_nodes, holes=0):
    markers = [api.BoundaryMarker(0, "DIRICHLET", "VECTOR_EDGE_ONLY", np.asarray(d), 0.0, "outer_faces"),
               api.BoundaryMarker(1, "DIRICHLET", "SCALAR_ONLY", np.asarray(scalar_nodes), 0.0, "outer_potential")]
    markers += [api.BoundaryMarker(2 + h, "NEUMANN", "VECTOR_EDGE_ONLY", np.zeros((0, 2), np.int32), 0.0,
                                   f"hole_{h}") for h in range(holes)]
    return api.EMMeshData(xyz=xyz, tets=el, boundary_markers=markers, dof_type=dof_type)


def product(md, gauge):
    dm = api.EMDOFManager(md)
    dm.build()
    nf = dm.getNumFreeDOFs()
    if gauge != _abi.GAUGE_NONE:
        dm.applyTreeGauge(api.GaugeMode(gauge))
    return dm, nf


def cases():
    for name in MESHES:
        for pat in ("all_av", "cycle", "av_vector", "av_scalar"):
            for holes in (0, 2):
                for gauge in (False, True):
                    yield name, pat, holes, gauge


@pytest.mark.parametrize("name,pat,holes,gauge", list(cases()))
def test_oracle_and_product_bit_exact_to_reference(name, pat, holes, gauge):
    xyz, el, d = MESHES[name]
    dt = av_patterns(el.shape[0])[pat]
    bnd = np.unique(np.asarray(d).ravel()).astype(np.int32)[::2]
    key = f"{name}_{pat}_h{holes}_{'gauge' if gauge else 'free'}"
    g = _abi.GAUGE_REF if gauge else _abi.GAUGE_NONE
    o = O.dof_build_av(el, dt, d, bnd, gauge=g, n_holes=holes, n_nodes=len(xyz))
    np.testing.assert_array_equal(o["l2g"], FIX[key])
    assert (o["n_free"], o["n_dofs"]) == (COUNTS[key]["n_free"], COUNTS[key]["n_dofs"])
    dm, nf = product(mesh_data(xyz, el, d, dt, bnd, holes), g)
    np.testing.assert_array_equal(dm.getElemLocalToGlobal(), FIX[key])
    assert (nf, dm.getNumFreeDOFs()) == (COUNTS[key]["n_free"], COUNTS[key]["n_dofs"])


@pytest.mark.parametrize("kind,n,seed", [("tet", 5, 1), ("tet", 8, 2), ("hex", 4, 3), ("hex", 5, 4)])
@pytest.mark.parametrize("gauge", [_abi.GAUGE_NONE, _abi.GAUGE_REF, _abi.GAUGE_BOUNDARY_FIRST])
def test_random_dof_types_match_oracle(kind, n, seed, gauge):
    if kind == "tet":
        m = mesh.random_instance(n, seed)
        xyz, el, d = m.xyz, m.tets, m.dirichlet
    else:
        xyz, el, d = mesh.hex_topology(n)
    rng = np.random.default_rng(seed)
    dt = rng.integers(0, 3, el.shape[0]).astype(np.int32)
    bnd = np.unique(np.asarray(d).ravel()).astype(np.int32)
    sd = rng.choice(bnd, size=len(bnd) // 2, replace=False)
    dm, nf = product(mesh_data(xyz, el, d, dt, sd), gauge)
    o = O.dof_build_av(el, dt, d, sd, gauge=gauge, n_nodes=len(xyz))
    np.testing.assert_array_equal(dm.getElemLocalToGlobal(), o["l2g"])
    assert (nf, dm.getNumFreeDOFs(), dm.getNumScalarFreeDOFs()) == (o["n_free"], o["n_dofs"], o["n_scalar_free"])


@pytest.mark.parametrize("gauge", [_abi.GAUGE_NONE, _abi.GAUGE_REF])
def test_all_mixed_av_is_scalar_block_then_shifted_edge_map(gauge):
    """With every element MIXED_AV the edge part is the edge-only map shifted
    past the free scalar DOFs, and the scalar part ranks the free nodes."""
    m = mesh.plain_small(4)
    bnd = np.unique(m.dirichlet.ravel()).astype(np.int32)
    dm, _ = product(mesh_data(m.xyz, m.tets, m.dirichlet, ["MIXED_AV"] * m.tets.shape[0], bnd), gauge)
    ns = dm.getNumScalarFreeDOFs()
    interior = np.setdiff1d(np.arange(m.n_nodes), bnd)
    assert ns == interior.size
    rows = dm.getElemLocalToGlobal()
    rank = np.full(m.n_nodes, -1)
    rank[interior] = np.arange(interior.size)
    np.testing.assert_array_equal(rows[:, :4], rank[m.tets])
    vec = O.dof_build(m.tets, m.dirichlet, gauge=gauge)
    np.testing.assert_array_equal(rows[:, 4:], np.where(vec["l2g"] < 0, -1, vec["l2g"] + ns))
    assert dm.getNumFreeDOFs() == ns + vec["n_dofs"]
    lst = dm.getElemLocalToGlobalList()
    assert all(len(r) == 10 for r in lst)


def test_scalar_only_mesh_has_no_edge_dofs():
    xyz, hexes, d = mesh.hex_topology(3)
    dm, nf = product(mesh_data(xyz, hexes, d, [0] * hexes.shape[0], []), _abi.GAUGE_REF)
    rows = dm.getElemLocalToGlobal()
    assert np.all(rows[:, 8:] == _abi.DOF_ABSENT)
    assert nf == dm.getNumFreeDOFs() == dm.getNumScalarFreeDOFs() == len(xyz)
    assert [len(r) for r in dm.getElemLocalToGlobalList()] == [8] * hexes.shape[0]


def test_invalid_dof_type_and_arguments_are_rejected():
    L = _abi.lib()
    m = mesh.plain_small(2)
    xyz = np.ascontiguousarray(m.xyz)
    tets = np.ascontiguousarray(m.tets, np.int32)
    d = np.ascontiguousarray(m.dirichlet, np.int32)
    h = C.c_void_p()
    _abi.check(L.emg_mesh_create(xyz.shape[0], _abi.ptr(xyz), tets.shape[0], _abi.ptr(tets), None, d.shape[0],
                                 _abi.ptr(d), 0, C.byref(h)), "emg_mesh_create")
    try:
        bad = np.full(tets.shape[0], 2, np.int32)
        bad[3] = 7
        assert L.emg_dof_build_av(h, _abi.ptr(bad), 0, None, _abi.GAUGE_REF, None, None, None, None) \
            == _abi.EMG_INVALID_INPUT
        assert b"element 3" in L.emg_last_error()
        assert L.emg_dof_build_av(h, None, 0, None, 5, None, None, None, None) == _abi.EMG_INVALID_INPUT
        assert L.emg_dof_build_av(h, None, 2, None, _abi.GAUGE_REF, None, None, None, None) \
            == _abi.EMG_INVALID_INPUT
        assert L.emg_dof_build_av(None, None, 0, None, _abi.GAUGE_REF, None, None, None, None) \
            == _abi.EMG_INVALID_INPUT
        # NULL dof_type = all MIXED_AV; node IDs outside the mesh constrain nothing
        ns, nd = C.c_int64(), C.c_int64()
        far = np.array([-5, 10 ** 6], np.int32)
        assert L.emg_dof_build_av(h, None, 2, _abi.ptr(far), _abi.GAUGE_REF, None, C.byref(ns), None,
                                  C.byref(nd)) == _abi.EMG_SUCCESS
        assert ns.value == m.n_nodes
    finally:
        L.emg_mesh_destroy(h)
