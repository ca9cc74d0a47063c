"""Failure paths of the GPU solvers, made on the host (no GPU fault).

* A right-hand side holding NaN: the reference's CGSolver / BiCGSTABSolver
  have no finiteness check (iterative_solvers.cpp:424-503, :869-1118), so
  every comparison with NaN is false and the solve runs to max_iter with
  MAX_ITER_REACHED; the GPU solvers follow the same rules, so statuses and
  iteration counts equal the oracle's.
* The bounded grid-barrier wait of the fused CG update: a test hook lowers
  its poll limit to zero, so the blocks that wait give up at once, raise
  the error flag and the solve ends with EMG_ERR_TIMEOUT; the context stays
  usable and the next solve (limit restored) converges.
"""
import ctypes as C

import numpy as np
import pytest

from emagddm_b200 import _abi, mesh
from oracle import oracle as O
from tests.helpers import System, lib, oracle_system, solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["cg", "bicgstab"])
@pytest.mark.parametrize("pc", [0, 1])
def test_nan_rhs_follows_reference_rules(kind, pc):
    m = mesh.plain_small(4)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    s = System(m, l2g)
    rp, col, kv, _, rhs = oracle_system(m, l2g)
    b = rhs.copy()
    b[3] = np.nan
    x, out = solve(s.matrix(0), b, kind, tol=1e-8, max_iter=40, precond=pc)
    fn = O.pcg if kind == "cg" else O.bicgstab
    _, st, it, res = fn(rp, col, kv, b, tol=1e-8, max_iter=40, precond=pc)
    assert out.status == st
    assert out.iterations == it
    assert np.isnan(out.residual_norm) == np.isnan(res)


def test_grid_barrier_wait_runs_out_with_timeout_status():
    m = mesh.plain_scale(24)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    s = System(m, l2g)
    n = int(l2g.max()) + 1
    cfg = _abi.KrylovConfig(1e-8, 5000, _abi.PRECOND_JACOBI)
    x = np.empty(n)
    try:
        _abi.check(lib().emg_test_set_barrier_spins(0), "emg_test_set_barrier_spins")
        out = _abi.Result()
        rc = lib().emg_system_solve(s.h, 0, C.byref(cfg), _abi.ptr(x), 0, None, C.byref(out))
        assert rc == out.status == _abi.EMG_ERR_TIMEOUT, (rc, out.status, lib().emg_last_error())
        assert out.iterations <= 3
    finally:
        _abi.check(lib().emg_test_set_barrier_spins(-1), "emg_test_set_barrier_spins")
    out = _abi.Result()
    rc = lib().emg_system_solve(s.h, 0, C.byref(cfg), _abi.ptr(x), 0, None, C.byref(out))
    assert rc == out.status == _abi.EMG_SUCCESS
    rp, col, kv, _, rhs = oracle_system(m, l2g)
    _, st, it, _ = O.pcg(rp, col, kv, rhs, tol=1e-8, max_iter=5000)
    assert abs(out.iterations - it) <= max(3, 0.15 * it)


def test_singular_system_factor_reports_numerical_error():
    """The direct backend on the ungauged curl-curl system (GAUGE_NONE: the
    discrete gradients of the interior nodes are in the kernel of K): the
    multifrontal Cholesky meets round-off-sized pivots and reports
    NUMERICAL_ERROR instead of returning a NaN or garbage solution; a solve
    without a successful factorization is INVALID_INPUT."""
    from emagddm_b200 import fetidp
    m = mesh.plain_scale(6)
    ds = fetidp.DirectSolver(m, gauge=_abi.GAUGE_NONE)
    assert ds.factor() == _abi.EMG_NUMERICAL_ERROR
    assert b"pivot" in lib().emg_last_error()
    _, rc, _ = ds.solve()
    assert rc == _abi.EMG_INVALID_INPUT
    # the same mesh gauged is regular: the factor succeeds and solves
    ok = fetidp.DirectSolver(m)
    assert ok.factor() == 0
    _, rc, out = ok.solve(tol=1e-12)
    assert rc == 0 and out.residual_norm < 1e-12
