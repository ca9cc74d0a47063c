"""Mixed-type meshes on the GPU through the C ABI against the oracle: one
symbolic phase over the 12-slot rows, one element-terms launch per type and
one gather; K, M, F to 1e-12 of the matrix scale with every flag, exact
symmetry, bit-exact patterns, discrete gradients in the kernel of the GPU
matrix, and Jacobi-PCG solutions to 1e-8 of the oracle's."""
import numpy as np
import pytest
import scipy.sparse as sp

from emagddm_b200 import _abi, mesh
from oracle import oracle as O
from tests.helpers import System, oracle_system, solve

pytestmark = pytest.mark.gpu
TOL = 1e-12
LAYOUTS = [("hex_prism", mesh.mixed_hex_prism), ("prism_tet", mesh.mixed_prism_tet),
           ("hex_pyramid_prism", mesh.mixed_hex_pyramid_prism)]


def close(a, b, tol=TOL):
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name,make", LAYOUTS)
@pytest.mark.parametrize("n,amp", [(4, 0.0), (6, 0.25)])
@pytest.mark.parametrize("gauge", [O.GAUGE_REF, O.GAUGE_NONE])
def test_stiffness_and_source_match_oracle(name, make, n, amp, gauge):
    m = make(n, small=False)
    m = mesh.perturbed(m, amp, seed=n) if amp else m
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=gauge)["l2g"]
    s = System(m, l2g)
    rp, col, kv, _, rhs = s.export()
    orp, ocol, okv, _, orhs = oracle_system(m, l2g)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert close(kv, okv)
    assert close(rhs, orhs) or np.abs(rhs - orhs).max() <= 1e-15
    A = sp.csr_matrix((kv, col, rp))
    assert (A != A.T).nnz == 0


@pytest.mark.parametrize("name,make", LAYOUTS)
@pytest.mark.parametrize("flags", [_abi.FLAG_MASS, _abi.FLAG_MASS | _abi.FLAG_NO_EDGE_SIGNS,
                                   _abi.FLAG_MASS | _abi.FLAG_PIOLA_LITERAL])
def test_flags_match_oracle(name, make, flags):
    m = mesh.perturbed(make(4, small=False), 0.2, seed=7)
    sigma = np.array([2.0, 5.8])
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    s = System(m, l2g, flags=flags, sigma=sigma)
    _, _, kv, mv, rhs = s.export()
    _, _, okv, omv, orhs = oracle_system(m, l2g, flags=flags, sigma=sigma)
    assert close(kv, okv) and close(mv, omv) and close(rhs, orhs)


@pytest.mark.parametrize("name,make", LAYOUTS)
def test_gradients_in_kernel_of_gpu_matrix(name, make):
    m = mesh.perturbed(make(6), 0.25, seed=4)
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_NONE)
    s = System(m, o["l2g"])
    rp, col, kv, _, _ = s.export()
    phi = np.random.default_rng(0).standard_normal(m.n_nodes)
    phi[np.unique(m.dirichlet)] = 0.0
    _, en = O.edge_ids(m.tets)
    g = np.zeros(o["n_dofs"])
    ok = o["edge_dof"] >= 0
    g[o["edge_dof"][ok]] = (phi[en[:, 1]] - phi[en[:, 0]])[ok]
    Kg = O.spmv(rp.astype(np.int64), col, kv, g)
    assert np.abs(Kg).max() <= 1e-12 * np.abs(kv).max() * np.abs(g).max()


@pytest.mark.parametrize("name,make", LAYOUTS)
def test_pcg_matches_oracle(name, make):
    m = mesh.perturbed(make(8, small=False), 0.2, seed=9)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    s = System(m, l2g)
    orp, ocol, okv, _, orhs = oracle_system(m, l2g)
    assert np.abs(orhs).max() > 1e-6
    x, out = solve(s.matrix(0), orhs, "cg", tol=1e-10, max_iter=50000, precond=1)
    xo, st, it, res = O.pcg(orp, ocol, okv, orhs, tol=1e-10, max_iter=50000, precond=1)
    assert out.status == st == 0
    assert abs(out.iterations - it) <= max(2, it // 50)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)


def test_tet_only_flag_is_rejected():
    m = mesh.mixed_prism_tet(3)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    with pytest.raises(_abi.EmgError):
        System(m, l2g, flags=_abi.FLAG_QUAD3_LITERAL)


@pytest.mark.parametrize("name,make", LAYOUTS)
def test_fetidp_and_direct_match_monolithic_oracle(name, make):
    from emagddm_b200 import fetidp
    m = mesh.perturbed(make(8, small=False), 0.2, seed=5)
    part = mesh.jittered_partition(m, 2)
    fd = fetidp.FetiDP(m, part, 8)
    assert fd.factor() == _abi.EMG_SUCCESS, _abi.lib().emg_last_error()
    x, rc, out = fd.solve(tol=1e-10, max_iter=2000, precond=2)
    assert rc == _abi.EMG_SUCCESS, (rc, _abi.lib().emg_last_error())
    rp, col, kv, _, rhs = oracle_system(m, fd.map.l2g)
    xo, st, it, res = O.pcg(rp, col, kv, rhs, tol=1e-13, max_iter=50000, precond=1)
    assert np.linalg.norm(xo) > 1e-6
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
    ds = fetidp.DirectSolver(m)
    assert ds.factor() == _abi.EMG_SUCCESS, _abi.lib().emg_last_error()
    xd, rc, out = ds.solve(tol=1e-12)
    assert rc == _abi.EMG_SUCCESS
    rp, col, kv, _, rhs = oracle_system(m, ds.l2g)
    xo, st, it, res = O.pcg(rp, col, kv, rhs, tol=1e-13, max_iter=50000, precond=1)
    assert np.linalg.norm(xd - xo) <= 1e-8 * np.linalg.norm(xo)
