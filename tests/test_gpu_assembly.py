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
