"""GPU assembly (symbolic pattern + numeric K, M, F) against the oracle and
the reference's golden pattern.

Tolerances: the CSR pattern is compared bit-exactly; values are compared
with |gpu - oracle| <= 1e-12 * max|oracle| entry-wise (the FP64 element-matrix
bar of the solve path); K must be exactly symmetric."""
import os

import numpy as np
import pytest

from emagddm_b200 import _abi, mesh
from oracle import oracle as O
from tests.helpers import System, oracle_system

pytestmark = pytest.mark.gpu
TOL = 1e-12
FIX = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.npz"))


def close(a, b, tol=TOL):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= tol * scale


def maps(m, gauge=O.GAUGE_REF):
    return O.dof_build(m.tets, m.dirichlet, gauge=gauge)["l2g"]


@pytest.mark.parametrize("n", [3, 4])
def test_pattern_bit_exact_to_reference(n):
    m = mesh.plain_small(n)
    s = System(m, maps(m))
    rp, col, _, _, _ = s.export()
    np.testing.assert_array_equal(rp, FIX[f"n{n}_pattern_row_ptr"])
    np.testing.assert_array_equal(col, FIX[f"n{n}_pattern_col"])


CASES = [("small", 2), ("small", 4), ("small", 8), ("scale", 6), ("scale", 10), ("rand", 7)]


def make(kind, n):
    if kind == "small":
        return mesh.plain_small(n)
    if kind == "scale":
        return mesh.plain_scale(n)
    return mesh.random_instance(n, seed=11)


@pytest.mark.parametrize("kind,n", CASES)
@pytest.mark.parametrize("gauge", [O.GAUGE_REF, O.GAUGE_NONE, O.GAUGE_BOUNDARY_FIRST])
def test_stiffness_and_source_match_oracle(kind, n, gauge):
    m = make(kind, n)
    l2g = maps(m, gauge)
    s = System(m, l2g)
    rp, col, kv, _, rhs = s.export()
    orp, ocol, okv, _, orhs = oracle_system(m, l2g)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert close(kv, okv)
    assert close(rhs, orhs) or np.abs(orhs).max() == 0.0
    # exact symmetry
    import scipy.sparse as sp
    A = sp.csr_matrix((kv, col, rp))
    assert (A != A.T).nnz == 0


@pytest.mark.parametrize("flags", [_abi.FLAG_MASS, _abi.FLAG_MASS | _abi.FLAG_NO_EDGE_SIGNS,
                                   _abi.FLAG_MASS | _abi.FLAG_PIOLA_LITERAL,
                                   _abi.FLAG_MASS | _abi.FLAG_QUAD3_LITERAL, _abi.FLAG_NO_EDGE_SIGNS])
def test_flags_match_oracle(flags):
    m = mesh.plain_scale(5)
    sigma = np.array([2.0, 5.8])
    l2g = maps(m)
    s = System(m, l2g, flags=flags, sigma=sigma)
    rp, col, kv, mv, rhs = s.export()
    orp, ocol, okv, omv, orhs = oracle_system(m, l2g, flags=flags, sigma=sigma)
    assert close(kv, okv)
    assert close(rhs, orhs)
    if flags & _abi.FLAG_MASS:
        assert close(mv, omv)


def fan_mesh(k=40):
    """k tets around the axis edge (0,0,0)-(0,0,1): that edge's row has
    2k + 3 columns, longer than the shared-memory rows of the gather kernel."""
    ang = np.linspace(0.0, 2 * np.pi, k, endpoint=False)
    ring = np.stack([np.cos(ang), np.sin(ang), 0.5 + 0.1 * np.sin(3 * ang)], axis=1)
    xyz = np.vstack([[0.0, 0.0, 0.0], [0.0, 0.0, 1.0], ring])
    tets = np.array([[0, 1, 2 + a, 2 + (a + 1) % k] for a in range(k)], np.int32)
    mat = (np.arange(k) % 2).astype(np.int32)
    src = [mesh.Source(mesh.SRC_BOX, (0.0, 0.0, 1.0), (-2.0, 2.0, -2.0, 2.0, -1.0, 2.0))]
    return mesh.CubeMesh(n=0, xyz=xyz, tets=tets, material=mat, dirichlet=np.zeros((0, 2), np.int32),
                         nu=np.array([1.0, 0.25]), sigma=np.array([1.0, 3.0]), sources=src, name="fan")


@pytest.mark.parametrize("flags", [0, _abi.FLAG_MASS])
def test_long_rows_match_oracle(flags):
    m = fan_mesh()
    l2g = maps(m, O.GAUGE_NONE)
    s = System(m, l2g, flags=flags)
    rp, col, kv, mv, rhs = s.export()
    assert np.diff(rp).max() > 64
    orp, ocol, okv, omv, orhs = oracle_system(m, l2g, flags=flags)
    np.testing.assert_array_equal(col, ocol)
    assert close(kv, okv) and close(rhs, orhs)
    if flags:
        assert close(mv, omv)


def test_two_local_edges_on_one_column_match_oracle():
    """A DOF map that sends two edges of one tet to the same column (merged
    DOFs): both terms land on that entry, in the element loop's order."""
    m = mesh.plain_scale(4)
    l2g = maps(m, O.GAUGE_NONE).reshape(-1, 6).copy()
    for t in (0, 7, 23):  # merge local edges 0 and 5 of a few tets, everywhere they occur
        a, b = l2g[t, 0], l2g[t, 5]
        l2g[l2g == b] = a
    l2g = l2g.ravel()
    used = np.unique(l2g[l2g >= 0])
    remap = -np.ones(int(l2g.max()) + 1, np.int64)
    remap[used] = np.arange(used.size)
    l2g = np.where(l2g >= 0, remap[np.maximum(l2g, 0)], -1).astype(np.int32)
    s = System(m, l2g, flags=_abi.FLAG_MASS, sigma=np.array([2.0, 5.8]))
    rp, col, kv, mv, rhs = s.export()
    orp, ocol, okv, omv, orhs = oracle_system(m, l2g, flags=_abi.FLAG_MASS, sigma=np.array([2.0, 5.8]))
    np.testing.assert_array_equal(col, ocol)
    assert close(kv, okv) and close(mv, omv) and close(rhs, orhs)


def test_deterministic_and_reassembly():
    m = mesh.plain_scale(8)
    s = System(m, maps(m))
    a = s.export()
    s.nu = s.nu * 2.0
    s.assemble()
    b = s.export()
    np.testing.assert_array_equal(b[2], 2.0 * a[2])  # K scales exactly with nu (power of 2)
    s.nu = s.nu / 2.0
    s.assemble()
    c = s.export()
    np.testing.assert_array_equal(a[2], c[2])
    np.testing.assert_array_equal(a[4], c[4])


def test_invalid_material_rejected():
    m = mesh.plain_small(2)
    s = System(m, maps(m))
    s.nu = np.array([-1.0])
    with pytest.raises(_abi.EmgError):
        s.assemble()


def test_transient_operator_and_bicgstab():
    """K + M/dt (eddy-current time step) on K's pattern, solved with BiCGSTAB
    and CG, against the oracle's assembly and solvers."""
    import ctypes as C

    from tests.helpers import lib, solve
    m = mesh.plain_scale(6)
    sigma = np.array([1.0, 5.0])
    l2g = maps(m)
    s = System(m, l2g, flags=_abi.FLAG_MASS, sigma=sigma)
    dt = 0.05
    h = C.c_void_p()
    _abi.check(lib().emg_system_combine(s.h, 1.0, 1.0 / dt, C.byref(h)), "combine")
    try:
        orp, ocol, okv, omv, orhs = oracle_system(m, l2g, flags=_abi.FLAG_MASS, sigma=sigma)
        A = okv + omv / dt
        import torch
        x = np.random.default_rng(3).normal(size=orhs.size)
        xd = torch.tensor(x, device="cuda")
        yd = torch.empty_like(xd)
        _abi.check(lib().emg_spmv(h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), None), "spmv")
        yo = O.spmv(orp, ocol, A, x)
        assert np.abs(yd.cpu().numpy() - yo).max() <= 1e-12 * np.abs(yo).max()
        for kind, pc in (("bicgstab", 0), ("cg", 1)):
            x, out = solve(h, orhs, kind, tol=1e-11, max_iter=5000, precond=pc)
            fn = O.bicgstab if kind == "bicgstab" else O.pcg
            xo, st, it, _ = fn(orp, ocol, A, orhs, tol=1e-11, max_iter=5000, precond=pc)
            assert out.status == st == 0
            assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
    finally:
        lib().emg_csr_destroy(h)
    # without a mass matrix the combination is refused
    s2 = System(m, l2g)
    h2 = C.c_void_p()
    assert lib().emg_system_combine(s2.h, 1.0, 1.0, C.byref(h2)) == _abi.EMG_INVALID_INPUT
