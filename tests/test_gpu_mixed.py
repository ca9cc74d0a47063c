"""Mixed-precision factor (EMG_FLAG_FACTOR_TF32): the contraction tiles of the
FETI-DP / direct factorizations on the tcgen05 tensor cores in two-term TF32
with FP32 accumulation, FP64 refinement on the true residual.

* The tile itself against FP64 products: |error| <= 4e-6 x sum |a_ik b_jk|
  (about 22 significant bits per product plus FP32 accumulation), rows and
  columns outside the tile untouched.
* FETI-DP and the direct solver with the mixed factor reach the same
  tolerances as the FP64 factor and agree with the oracle's monolithic FP64
  solve to 1e-8 (1e-9 for the direct solver), the solve path's bar.
"""
import ctypes as C

import numpy as np
import pytest

from emagddm_b200 import _abi, fetidp, mesh
from oracle import oracle as O
from tests.helpers import lib, oracle_system

pytestmark = pytest.mark.gpu
FLAG_TF32 = 16


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


@pytest.mark.parametrize("mr,mc,k,scale", [(128, 128, 64, 0), (128, 128, 300, 0), (77, 128, 5, 0),
                                           (128, 33, 16, 3), (1, 1, 1, 0), (90, 100, 0, 0), (128, 128, 129, 6)])
def test_tc_tile_matches_fp64(mr, mc, k, scale):
    import torch
    rng = np.random.default_rng(mr * 7 + mc * 3 + k)
    lda, ldb, ldc = mr + 5, mc + 3, mr + 9
    # column-major storage: (k, ld) in C order is (ld, k) column-major
    # (at least one column allocated: k = 0 still passes valid pointers)
    A = rng.standard_normal((max(k, 1), lda))
    B = rng.standard_normal((max(k, 1), ldb))
    if scale:  # rows spanning +-scale decades
        A *= 10.0 ** rng.uniform(-scale, scale, size=(1, lda))
        B *= 10.0 ** rng.uniform(-scale, scale, size=(1, ldb))
    Cm = rng.standard_normal((mc, ldc))
    dA, dB, dC = _dev(A), _dev(B), _dev(Cm)
    rc = lib().emg_test_tc_tile(mr, mc, k, C.c_void_p(dA.data_ptr()), lda, C.c_void_p(dB.data_ptr()), ldb,
                                C.c_void_p(dC.data_ptr()), ldc, None)
    torch.cuda.synchronize()
    assert rc == _abi.EMG_SUCCESS, lib().emg_last_error()
    out = dC.cpu().numpy()
    a, b = A[:k, :mr].T, B[:k, :mc].T          # (mr, k), (mc, k)
    want = Cm[:mc, :mr] - (a @ b.T).T           # C stored (mc, ldc): [col, row]
    bound = 4e-6 * (np.abs(a) @ np.abs(b).T).T + 1e-300
    assert np.all(np.abs(out[:mc, :mr] - want) <= bound), np.max(np.abs(out[:mc, :mr] - want) / bound)
    np.testing.assert_array_equal(out[:mc, mr:], Cm[:mc, mr:])   # padding rows of C
    np.testing.assert_array_equal(out[mc:, :], Cm[mc:, :])


def test_tc_tile_rejects_bad_sizes():
    rc = lib().emg_test_tc_tile(129, 8, 4, None, 129, None, 8, None, 129, None)
    assert rc == _abi.EMG_INVALID_INPUT


def _monolithic(m, l2g, tol=1e-12):
    rp, col, kv, _, rhs = oracle_system(m, l2g)
    x, st, it, res = O.pcg(rp, col, kv, rhs, tol=tol, max_iter=50000, precond=1)
    assert st == 0 or (st == _abi.EMG_NUMERICAL_ERROR and res < 10 * tol), (st, res)
    return x


@pytest.mark.parametrize("kind,n,parts", [("scale", 8, 2), ("small", 16, 4), ("scale", 16, 2)])
def test_mixed_factor_fetidp_matches_oracle(kind, n, parts):
    m = mesh.plain_scale(n) if kind == "scale" else mesh.plain_small(n)
    part = mesh.jittered_partition(m, parts)
    fd = fetidp.FetiDP(m, part, parts ** 3)
    assert fd.factor(flags=FLAG_TF32) == _abi.EMG_SUCCESS, lib().emg_last_error()
    # residuals well below the solution bar on both sides, so that the
    # comparison measures the solvers, not their stopping points
    x, rc, out = fd.solve(tol=1e-11, max_iter=5000)
    assert rc == _abi.EMG_SUCCESS, (rc, lib().emg_last_error())
    assert out.residual_norm <= 1e-11
    xo = _monolithic(m, fd.map.l2g, tol=1e-13)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
    # the FP64 factor of the same plan gives the same solution
    assert fd.factor() == _abi.EMG_SUCCESS
    x64, rc, _ = fd.solve(tol=1e-11, max_iter=5000)
    assert rc == 0 and np.linalg.norm(x - x64) <= 1e-8 * np.linalg.norm(x64)


@pytest.mark.parametrize("n", [10, 14])
def test_mixed_factor_direct_matches_oracle(n):
    m = mesh.plain_scale(n)
    ds = fetidp.DirectSolver(m)
    assert ds.factor(flags=FLAG_TF32) == 0, lib().emg_last_error()
    x, rc, out = ds.solve(tol=1e-12, passes=30)
    assert rc == 0, (rc, lib().emg_last_error())
    assert out.residual_norm <= 1e-12
    xo = _monolithic(m, ds.l2g)
    assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)


def test_factor_kinds_alternate_with_graph_replay():
    """FP64 and TF32 factorizations alternating on one solver: each kind runs
    eagerly once before it is captured as a graph (its kernels' shared-memory
    limits are set by the eager run), so no capture fails and every
    factorization gives the solution of its kind bit for bit."""
    m = mesh.plain_scale(8)
    part = mesh.jittered_partition(m, 2)
    fd = fetidp.FetiDP(m, part, 8)
    xs = {0: [], FLAG_TF32: []}
    for flags in (0, 0, FLAG_TF32, FLAG_TF32, 0, FLAG_TF32):
        assert fd.factor(flags=flags) == _abi.EMG_SUCCESS, lib().emg_last_error()
        assert b"capture" not in lib().emg_last_error()
        x, rc, _ = fd.solve(tol=1e-11, max_iter=5000)
        assert rc == _abi.EMG_SUCCESS, (rc, lib().emg_last_error())
        xs[flags].append(x)
    for kind in xs.values():
        for x in kind[1:]:
            np.testing.assert_array_equal(x, kind[0])
    assert np.linalg.norm(xs[FLAG_TF32][0] - xs[0][0]) <= 1e-8 * np.linalg.norm(xs[0][0])
