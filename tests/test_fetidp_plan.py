"""Partitioned tree-cotree gauge and the FETI-DP symbolic plan (host only, no
GPU): the gauge must be complete (same unknown count as a tree spanning every
interior node), the box partition of the cube must need exactly its wire-basket
cotree edges as primal DOFs, and the plan's own index check must pass for box,
slab, single-subdomain and scattered partitions."""
import numpy as np
import pytest

from emagddm_b200 import fetidp, mesh
from oracle import oracle as O


def scattered(m, k):
    # tets dealt round-robin over k subdomains by hex: every subdomain is a
    # scatter of disconnected hexes, so most edges are shared by >= 3
    return ((np.arange(m.n_tets) // 6) % k).astype(np.int32)


@pytest.mark.parametrize("n,parts", [(4, 2), (8, 2), (12, 3), (16, 4)])
def test_partitioned_gauge_is_complete(n, parts):
    m = mesh.plain_scale(n)
    part = mesh.jittered_partition(m, parts)
    pm = fetidp.partitioned_dofmap(m, part, parts ** 3)
    bf = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_BOUNDARY_FIRST)
    assert pm.n_dofs == bf["n_dofs"]
    assert pm.n_parts == parts ** 3
    # reduced DOFs are numbered in ascending edge ID, -1 elsewhere
    kept = pm.edge_dof[pm.edge_dof >= 0]
    np.testing.assert_array_equal(kept, np.arange(pm.n_dofs))
    free = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_NONE)
    assert pm.n_free == free["n_dofs"]


def test_box_partition_primal_is_the_wire_basket():
    m = mesh.plain_small(16)
    part = mesh.jittered_partition(m, 4)
    pm = fetidp.partitioned_dofmap(m, part, 64)
    assert pm.n_primal_fix == 0
    assert pm.primal.sum() == 81
    # every primal DOF is shared by >= 3 subdomains
    sets = {}
    for t in range(m.n_tets):
        for g in pm.l2g[t]:
            if g >= 0:
                sets.setdefault(int(g), set()).add(int(part[t]))
    for g in np.flatnonzero(pm.primal):
        assert len(sets[int(g)]) >= 3


def test_single_subdomain_has_no_interface():
    m = mesh.plain_small(6)
    info = fetidp.plan_info(m, np.zeros(m.n_tets, np.int32), 1)
    assert info["n_lambda"] == 0 and info["n_coarse"] == 0 and info["sum_nD"] == 0
    assert info["n_union"] == info["n_dofs"]


@pytest.mark.parametrize("case", ["slab2", "box8", "box64", "scattered3", "scattered5"])
def test_plan_validates(case):
    if case == "slab2":
        m = mesh.plain_scale(10)
        part = (mesh.centroids(m.xyz, m.tets)[:, 0] > 0.45).astype(np.int32)
        k = 2
    elif case == "box8":
        m = mesh.random_instance(12, 3)
        part, k = mesh.jittered_partition(m, 2), 8
    elif case == "box64":
        m = mesh.plain_scale(16)
        part, k = mesh.jittered_partition(m, 4, seed=5), 64
    else:
        k = int(case[-1])
        m = mesh.plain_small(6)
        part = scattered(m, k)
    info = fetidp.plan_info(m, part, k)  # raises if the plan check fails
    pm = fetidp.partitioned_dofmap(m, part, k)
    assert info["n_coarse"] == int(pm.primal.sum())
    # every DOF appears in the union once per subdomain that touches it
    copies = info["sum_nI"] + info["sum_nD"] + info["sum_nP"]
    assert copies == info["n_union"]
    assert info["sum_nD"] == 2 * info["n_lambda"]
    if case == "slab2":
        assert info["n_coarse"] == 0 and pm.n_primal_fix == 0


def test_bad_partition_rejected():
    m = mesh.plain_small(3)
    part = np.zeros(m.n_tets, np.int32)
    part[5] = 7
    with pytest.raises(RuntimeError, match="tet_part"):
        fetidp.partitioned_dofmap(m, part, 2)


@pytest.mark.parametrize("gauge", [O.GAUGE_REF, O.GAUGE_BOUNDARY_FIRST])
def test_direct_solver_plan_on_gauged_maps(gauge):
    # the direct solver analyses any map as one subdomain
    m = mesh.plain_scale(10)
    maph, mh, l2g, n = fetidp.gauged_map(m, gauge)
    info = np.zeros(len(fetidp.INFO_KEYS), np.int64)
    from emagddm_b200 import _abi
    _abi.check(_abi.lib().emg_fetidp_plan_info(mh.h, maph.h, _abi.ptr(info), len(info)), "plan_info")
    d = dict(zip(fetidp.INFO_KEYS, info))
    assert d["n_parts"] == 1 and d["n_lambda"] == 0 and d["n_coarse"] == 0
    assert d["n_dofs"] == n == d["n_union"] == d["sum_nI"]
    assert n == O.dof_build(m.tets, m.dirichlet, gauge=gauge)["n_dofs"]
