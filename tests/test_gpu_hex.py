"""HEX8_EDGE on the GPU through the C ABI against the oracle: the merged CSR
pattern bit-exact (and equal to the reference's golden pattern), K, M, F to
1e-12 of the matrix scale, exact symmetry, discrete gradients in the kernel
of the assembled K, Jacobi-PCG solutions to 1e-8, and the FETI-DP and direct
solvers on hexahedral meshes against the oracle's monolithic solve (1e-8)."""
import os

import numpy as np
import pytest

from emagddm_b200 import _abi, fetidp, mesh
from oracle import oracle as O
from tests.helpers import System, oracle_system, solve

pytestmark = pytest.mark.gpu
TOL = 1e-12
FIX = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_hex_fixtures.npz"))


def close(a, b, tol=TOL):
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)


def maps(m, gauge=O.GAUGE_REF):
    return O.dof_build(m.tets, m.dirichlet, gauge=gauge)["l2g"]


def test_hex_pattern_bit_exact_to_reference():
    m = mesh.hex_small(3)
    s = System(m, maps(m))
    rp, col, _, _, _ = s.export()
    np.testing.assert_array_equal(rp, FIX["hex_n3_pattern_row_ptr"])
    np.testing.assert_array_equal(col, FIX["hex_n3_pattern_col"])


CASES = [("small", 4, 0.0), ("scale", 6, 0.0), ("scale", 8, 0.25), ("small", 10, 0.2)]


def make(kind, n, amp):
    m = mesh.hex_small(n) if kind == "small" else mesh.hex_scale(n)
    return mesh.perturbed(m, amplitude=amp, seed=n) if amp > 0 else m


@pytest.mark.parametrize("kind,n,amp", CASES)
@pytest.mark.parametrize("gauge", [O.GAUGE_REF, O.GAUGE_NONE])
def test_hex_stiffness_and_source_match_oracle(kind, n, amp, gauge):
    m = make(kind, n, amp)
    l2g = maps(m, gauge)
    s = System(m, l2g)
    rp, col, kv, _, rhs = s.export()
    orp, ocol, okv, _, orhs = oracle_system(m, l2g)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert close(kv, okv)
    # symmetric source placements can leave F at rounding level (|F| < 1e-15)
    assert close(rhs, orhs) or (np.abs(orhs).max() < 1e-15 and np.abs(rhs).max() < 1e-15)
    import scipy.sparse as sp
    A = sp.csr_matrix((kv, col, rp))
    assert (A != A.T).nnz == 0


@pytest.mark.parametrize("flags", [_abi.FLAG_MASS, _abi.FLAG_MASS | _abi.FLAG_NO_EDGE_SIGNS,
                                   _abi.FLAG_MASS | _abi.FLAG_PIOLA_LITERAL, _abi.FLAG_NO_EDGE_SIGNS])
def test_hex_flags_match_oracle(flags):
    m = mesh.perturbed(mesh.hex_scale(5), amplitude=0.2, seed=1)
    sigma = np.array([2.0, 5.8])
    l2g = maps(m)
    s = System(m, l2g, flags=flags, sigma=sigma)
    _, _, kv, mv, rhs = s.export()
    _, _, okv, omv, orhs = oracle_system(m, l2g, flags=flags, sigma=sigma)
    assert close(kv, okv)
    assert close(rhs, orhs)
    if flags & _abi.FLAG_MASS:
        assert close(mv, omv)


def test_hex_gradients_in_kernel_of_gpu_matrix():
    m = mesh.perturbed(mesh.hex_scale(6), amplitude=0.25, seed=4)
    o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_NONE)
    s = System(m, o["l2g"])
    rp, col, kv, _, _ = s.export()
    rng = np.random.default_rng(0)
    phi = rng.standard_normal(m.n_nodes)
    phi[np.any((m.xyz < 1e-12) | (m.xyz > 1 - 1e-12), axis=1)] = 0.0
    _, en = O.edge_ids(m.tets)
    g = np.zeros(o["n_free"])
    ok = o["edge_dof"] >= 0
    g[o["edge_dof"][ok]] = ((phi[en[:, 1]] - phi[en[:, 0]]) / 4.0)[ok]
    Kg = O.spmv(rp.astype(np.int64), col, kv, g)
    assert np.abs(Kg).max() <= 1e-12 * np.abs(kv).max() * np.abs(g).max()


# On the unperturbed grid the `ref` tree takes every z-directed edge, so the
# z-directed coil current has no cotree test function and F vanishes; the
# solver cases use perturbed geometry, where F is far from rounding level.
@pytest.mark.parametrize("amp", [0.15, 0.3])
def test_hex_pcg_matches_oracle(amp):
    m = make("scale", 10, amp)
    l2g = maps(m)
    s = System(m, l2g)
    orp, ocol, okv, _, orhs = oracle_system(m, l2g)
    assert np.abs(orhs).max() > 1e-6
    x, out = solve(s.matrix(0), orhs, "cg", tol=1e-10, max_iter=20000, precond=1)
    xo, st, it, res = O.pcg(orp, ocol, okv, orhs, tol=1e-10, max_iter=20000, precond=1)
    assert out.status == st == 0
    assert abs(out.iterations - it) <= max(2, it // 50)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)


def monolithic(m, l2g):
    rp, col, kv, _, rhs = oracle_system(m, l2g)
    x, st, it, res = O.pcg(rp, col, kv, rhs, tol=1e-13, max_iter=50000, precond=1)
    assert st == 0 or (st == _abi.EMG_NUMERICAL_ERROR and res < 1e-12), (st, res)
    return x


@pytest.mark.parametrize("n,parts,amp", [(8, 2, 0.2), (12, 3, 0.25)])
def test_hex_fetidp_matches_monolithic_oracle(n, parts, amp):
    m = make("scale", n, amp)
    part = mesh.jittered_partition(m, parts)
    fd = fetidp.FetiDP(m, part, parts ** 3)
    assert fd.factor() == _abi.EMG_SUCCESS, _abi.lib().emg_last_error()
    for pc in (2, 3):
        x, rc, out = fd.solve(tol=1e-10, max_iter=2000, precond=pc)
        assert rc == _abi.EMG_SUCCESS, (rc, _abi.lib().emg_last_error())
        xo = monolithic(m, fd.map.l2g)
        assert np.linalg.norm(xo) > 1e-6
        assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
        assert out.residual_norm <= 1e-10


def test_hex_direct_solver_on_reference_gauge():
    m = make("scale", 10, 0.15)
    ds = fetidp.DirectSolver(m)
    assert ds.factor() == _abi.EMG_SUCCESS, _abi.lib().emg_last_error()
    x, rc, out = ds.solve(tol=1e-12)
    assert rc == _abi.EMG_SUCCESS, _abi.lib().emg_last_error()
    xo = monolithic(m, ds.l2g)
    assert np.linalg.norm(xo) > 1e-6
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
