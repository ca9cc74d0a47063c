"""Device DOF numbering (emg_dof_build_device) against the host numbering and
the oracle: Local2Global maps and counts bit-exact for every element type and
mixed meshes,
the `ref` gauge and none, full / partial / empty Dirichlet lists, hole
markers and meshes of several components; invalid input is rejected."""
import ctypes as C

import numpy as np
import pytest
import torch

from emagddm_b200 import _abi, mesh
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def device_map(elems, n_nodes, dirichlet, gauge, holes=0):
    L = _abi.lib()
    dev = torch.device("cuda", 0)
    e = torch.from_numpy(np.ascontiguousarray(elems, np.int32)).to(dev)
    d = torch.from_numpy(np.ascontiguousarray(dirichlet, np.int32).reshape(-1)).to(dev)
    epe = mesh.EDGES_OF_TYPE[mesh.TYPE_OF_NODES[elems.shape[1]]]
    l2g = torch.empty(epe * elems.shape[0], dtype=torch.int32, device=dev)
    ne, nf, nd = C.c_int64(), C.c_int64(), C.c_int64()
    rc = L.emg_dof_build_device(mesh.TYPE_OF_NODES[elems.shape[1]], n_nodes, elems.shape[0], e.data_ptr(),
                                len(dirichlet), d.data_ptr() if len(dirichlet) else None, holes, gauge,
                                l2g.data_ptr(), C.byref(ne), C.byref(nf), C.byref(nd), None)
    return rc, l2g.cpu().numpy().reshape(elems.shape[0], epe), ne.value, nf.value, nd.value


MESHES = [("tet", lambda: mesh.plain_scale(6)), ("tet_perturbed", lambda: mesh.perturbed(mesh.plain_scale(5), 0.2, 1)),
          ("random", lambda: mesh.random_instance(7, seed=3)), ("hex", lambda: mesh.hex_scale(5)),
          ("prism", lambda: mesh.prism_scale(5)), ("pyramid", lambda: mesh.pyramid_scale(4)),
          ("mixed_hex_prism", lambda: mesh.mixed_hex_prism(4)), ("mixed_prism_tet", lambda: mesh.mixed_prism_tet(4)),
          ("mixed_hex_pyramid_prism", lambda: mesh.perturbed(mesh.mixed_hex_pyramid_prism(4), 0.2, 2))]


@pytest.mark.parametrize("name,make", MESHES)
@pytest.mark.parametrize("gauge", [O.GAUGE_REF, O.GAUGE_NONE])
@pytest.mark.parametrize("which", ["full", "partial", "none"])
def test_device_numbering_matches_host(name, make, gauge, which):
    m = make()
    d = {"full": m.dirichlet, "partial": m.dirichlet[np.random.default_rng(2).permutation(len(m.dirichlet))[::3]],
         "none": np.zeros((0, 2), np.int32)}[which]
    for holes in ((0, 2) if gauge == O.GAUGE_REF else (0,)):
        rc, l2g, ne, nf, nd = device_map(m.tets, m.n_nodes, d, gauge, holes)
        assert rc == 0, _abi.lib().emg_last_error()
        o = O.dof_build(m.tets, d, gauge=gauge, n_holes=holes)
        np.testing.assert_array_equal(l2g, o["l2g"])
        assert (ne, nf, nd) == (o["n_edges"], o["n_free"], o["n_dofs"])


def test_several_components():
    a = mesh.plain_small(3)
    b = mesh.perturbed(mesh.plain_small(2), 0.2, 4)
    tets = np.vstack([a.tets, b.tets + a.n_nodes])
    d = np.vstack([a.dirichlet[::2], b.dirichlet[:9] + a.n_nodes])
    for dd in (d, d[len(a.dirichlet[::2]):], np.zeros((0, 2), np.int32)):
        rc, l2g, ne, nf, nd = device_map(tets, a.n_nodes + b.n_nodes, dd, O.GAUGE_REF)
        assert rc == 0
        o = O.dof_build(tets, dd, gauge=O.GAUGE_REF)
        np.testing.assert_array_equal(l2g, o["l2g"])
        assert nd == o["n_dofs"]


def test_invalid_input_is_rejected():
    m = mesh.plain_small(2)
    bad = m.tets.copy()
    bad[3, 1] = m.n_nodes + 5
    rc, *_ = device_map(bad, m.n_nodes, m.dirichlet, O.GAUGE_REF)
    assert rc == _abi.EMG_INVALID_INPUT
    rc, *_ = device_map(m.tets, m.n_nodes, m.dirichlet, O.GAUGE_BOUNDARY_FIRST)
    assert rc == _abi.EMG_INVALID_INPUT
