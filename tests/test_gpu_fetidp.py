"""FETI-DP on the GPU against the oracle's monolithic FP64 solve of the same
partition-gauged system (solution within 1e-8 relative) and its reported true
residual."""
import numpy as np
import pytest

from emagddm_b200 import _abi, fetidp, mesh
from oracle import oracle as O
from tests.helpers import oracle_system

pytestmark = pytest.mark.gpu

CASES = [("scale", 6, 2), ("scale", 8, 2), ("rand", 12, 2), ("small", 16, 4), ("scatter", 6, 3)]


def make(kind, n, parts):
    if kind == "scale":
        m = mesh.plain_scale(n)
    elif kind == "small":
        m = mesh.plain_small(n)
    else:
        m = mesh.random_instance(n, seed=11) if kind == "rand" else mesh.plain_scale(n)
    if kind == "scatter":
        return m, ((np.arange(m.n_tets) // 6) % parts).astype(np.int32), parts
    return m, mesh.jittered_partition(m, parts), parts ** 3


def monolithic(m, l2g):
    rp, col, kv, _, rhs = oracle_system(m, l2g)
    x, st, it, res = O.pcg(rp, col, kv, rhs, tol=1e-13, max_iter=50000, precond=1)
    # at 1e-13 the oracle's p.Ap < 1e-30 breakdown guard can fire once it has converged
    assert st == 0 or (st == _abi.EMG_NUMERICAL_ERROR and res < 1e-12), (st, res)
    return x, rhs


@pytest.mark.parametrize("kind,n,parts", CASES)
def test_fetidp_matches_monolithic_oracle(kind, n, parts):
    m, part, k = make(kind, n, parts)
    fd = fetidp.FetiDP(m, part, k)
    assert fd.factor() == _abi.EMG_SUCCESS, _abi.lib().emg_last_error()
    x, rc, out = fd.solve(tol=1e-10, max_iter=1000)
    assert rc == _abi.EMG_SUCCESS, (rc, _abi.lib().emg_last_error())
    xo, rhs = monolithic(m, fd.map.l2g)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
    assert out.residual_norm <= 1e-10
    st = fd.stats()
    assert st["iterations"] == out.iterations and st["residual"] == out.residual_norm


@pytest.mark.parametrize("precond", [0, 1, 2, 3])
def test_fetidp_preconditioners_agree(precond):
    m, part, k = make("scale", 8, 2)
    fd = fetidp.FetiDP(m, part, k)
    assert fd.factor() == 0
    x, rc, out = fd.solve(tol=1e-10, max_iter=3000, precond=precond)
    assert rc == 0, _abi.lib().emg_last_error()
    xo, _ = monolithic(m, fd.map.l2g)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
    _, rc, _ = fd.solve(precond=4)
    assert rc == _abi.EMG_INVALID_INPUT


def test_deluxe_beats_stiffness_on_a_coefficient_jump():
    # mu_r = 1000 block cutting through subdomains: deluxe keeps the count low
    m, part, k = make("scale", 16, 4)
    fd = fetidp.FetiDP(m, part, k)
    assert fd.factor() == 0
    _, rc1, o1 = fd.solve(tol=1e-10, precond=1)
    _, rc2, o2 = fd.solve(tol=1e-10, precond=2)
    assert rc1 == rc2 == 0
    assert o2.iterations * 2 < o1.iterations, (o1.iterations, o2.iterations)


def test_fetidp_refactor_and_iteration_limit():
    m, part, k = make("scale", 8, 2)
    fd = fetidp.FetiDP(m, part, k)
    assert fd.factor() == 0
    x1, rc, out1 = fd.solve(tol=1e-10)
    assert rc == 0
    # new materials on the same plan
    assert fd.factor(nu=np.array([1.0, 0.01])) == 0
    x2, rc, _ = fd.solve(tol=1e-10)
    assert rc == 0 and np.linalg.norm(x2 - x1) > 1e-3 * np.linalg.norm(x1)
    assert fd.factor() == 0
    x3, rc, _ = fd.solve(tol=1e-10)
    assert rc == 0 and np.linalg.norm(x3 - x1) <= 1e-12 * np.linalg.norm(x1)
    _, rc, out = fd.solve(tol=1e-14, max_iter=1)
    assert rc == _abi.EMG_MAX_ITER_REACHED and out.iterations == 1


def test_gauge_only_removes_gradients():
    """For a consistent right-hand side F = K_free y (y on every free edge), the
    partition-gauged FETI-DP solution, extended by zeros on the tree edges,
    solves the full ungauged curl-curl system: the gauge only fixes the
    gradient part, so B = curl A is the physical field."""
    m, part, k = make("scale", 8, 2)
    fd = fetidp.FetiDP(m, part, k)
    assert fd.factor() == 0
    free = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_NONE)
    n_free = int(free["n_dofs"])
    frp, fcol, fkv, _, _ = oracle_system(m, free["l2g"])
    y = np.random.default_rng(5).normal(size=n_free)
    Ffree = O.spmv(frp, fcol, fkv, y)
    free_of_edge = np.full(fd.map.edge_dof.size, -1, np.int64)
    free_of_edge[free["elem_edge"].ravel()] = free["l2g"].ravel()
    kept = np.flatnonzero(fd.map.edge_dof >= 0)
    b = np.empty(fd.map.n_dofs)
    b[fd.map.edge_dof[kept]] = Ffree[free_of_edge[kept]]
    x, rc, out = fd.solve_rhs(b, tol=1e-11, max_iter=2000)
    assert rc == 0, _abi.lib().emg_last_error()
    xfull = np.zeros(n_free)
    xfull[free_of_edge[kept]] = x[fd.map.edge_dof[kept]]
    r = Ffree - O.spmv(frp, fcol, fkv, xfull)
    assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(Ffree)


@pytest.mark.parametrize("kind,n", [("scale", 6), ("scale", 10), ("rand", 9), ("small", 12)])
def test_direct_solver_on_reference_gauge(kind, n):
    """Multifrontal GPU Cholesky of the reference-exact (ref-gauge) system
    against the oracle's monolithic solve."""
    m = {"scale": mesh.plain_scale, "small": mesh.plain_small}.get(kind, lambda k: mesh.random_instance(k, 11))(n)
    ds = fetidp.DirectSolver(m)
    assert ds.factor() == 0, _abi.lib().emg_last_error()
    x, rc, out = ds.solve(tol=1e-12)
    assert rc == 0, _abi.lib().emg_last_error()
    xo, rhs = monolithic(m, ds.l2g)
    assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)
    assert out.residual_norm <= 1e-12
    # a second right-hand side on the same factorization
    b2 = np.random.default_rng(1).normal(size=ds.n_dofs)
    x2, rc, out2 = ds.solve(b2, tol=1e-12)
    assert rc == 0 and out2.residual_norm <= 1e-12
    rp, col, kv, _, _ = oracle_system(m, ds.l2g)
    assert np.linalg.norm(b2 - O.spmv(rp, col, kv, x2)) <= 1e-11 * np.linalg.norm(b2)


def test_factor_graph_replay_matches_the_eager_factorization():
    """The first factorization of a plan runs eagerly, the second is captured
    as one CUDA graph, later ones replay it: the same kernels in the same
    order, so the solutions agree bit for bit (and a different material set
    between them is picked up by the replay)."""
    m, part, k = make("scale", 8, 2)
    fd = fetidp.FetiDP(m, part, k)
    xs = []
    for nu in (None, None, np.array([1.0, 0.01]), None):
        assert fd.factor(nu=nu) == 0, _abi.lib().emg_last_error()
        x, rc, _ = fd.solve(tol=1e-10, max_iter=1000)
        assert rc == 0
        xs.append(x)
    np.testing.assert_array_equal(xs[0], xs[1])
    np.testing.assert_array_equal(xs[0], xs[3])
    assert np.linalg.norm(xs[2] - xs[0]) > 1e-3 * np.linalg.norm(xs[0])
