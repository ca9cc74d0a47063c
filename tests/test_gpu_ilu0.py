"""The ILU0 preconditioner option of CGSolver / BiCGSTABSolver on the GPU.

The reference factors Eigen::IncompleteLUT (iterative_solvers.cpp:277-286);
the GPU factors ILU(0) on the matrix's pattern, so the iteration counts differ
and parity is on the converged solution:
* CG against the reference's own CGSolver with ILU0 (golden fixtures from
  the reference compiled here, tests/golden/make_golden.py --ilu0-only):
  SUCCESS and solutions within 1e-8 relative; iteration counts against the
  oracle's ILU(0) restatement (statuses too for BiCGSTAB, whose reference
  iteration stalls with ILU(0));
* against the FP64 oracle's monolithic solve at 16^3 (the 'plain method,
  small' system), through emg_system_solve: within 1e-8;
* ILU(0) of a tridiagonal matrix is its exact LU, so preconditioned CG
  converges in one iteration;
* a factorization that breaks down (zero pivot, missing diagonal) leaves the
  solve without a preconditioner, exactly as the reference's
  setup_preconditioner does: same status, iterations and x as NONE.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from emagddm_b200 import _abi, api, mesh
from oracle import oracle as O
from tests.helpers import HostCsr, System, lib, oracle_system, solve

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIX = np.load(os.path.join(GOLD, "reference_ilu0_fixtures.npz"))
COUNTS = json.load(open(os.path.join(GOLD, "reference_ilu0_counts.json")))
ILU0 = _abi.PRECOND_ILU0


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("tag", ["n4", "s6"])
def test_ilu0_cg_matches_reference_and_oracle(tag):
    rp, col, kv, b = FIX[f"{tag}_row_ptr"], FIX[f"{tag}_col"], FIX[f"{tag}_val"], FIX[f"{tag}_rhs"]
    A = HostCsr(rp.astype(np.int32), col, kv)
    assert COUNTS[f"{tag}_cg_ilu0"]["status"] == 0
    x, out = solve(A.h, b, "cg", tol=1e-10, max_iter=1000, precond=ILU0)
    assert out.status == _abi.EMG_SUCCESS and out.residual_norm < 1e-10
    assert rel(x, FIX[f"{tag}_cg_ilu0_x"]) <= 1e-8           # the reference's converged solution
    xo, st, it, _ = O.pcg(rp, col, kv, b, tol=1e-10, max_iter=1000, precond=ILU0)
    assert st == 0 and abs(out.iterations - it) <= max(3, 0.15 * it)   # the same ILU(0) iteration
    # a preconditioner that pays: fewer iterations than Jacobi on the same system
    _, oj = solve(A.h, b, "cg", tol=1e-10, max_iter=5000, precond=1)
    assert out.iterations < oj.iterations


@pytest.mark.parametrize("tag", ["n4", "s6"])
def test_ilu0_bicgstab_follows_the_reference_iteration(tag):
    """The reference's BiCGSTAB ILU0 iteration leaves p unpreconditioned and
    takes omega = z.t / t.t (iterative_solvers.cpp:1162-1191).  With its
    near-exact IncompleteLUT it converges here; with ILU(0) the same
    iteration stalls, on the GPU exactly as in the oracle's restatement."""
    rp, col, kv, b = FIX[f"{tag}_row_ptr"], FIX[f"{tag}_col"], FIX[f"{tag}_val"], FIX[f"{tag}_rhs"]
    A = HostCsr(rp.astype(np.int32), col, kv)
    x, out = solve(A.h, b, "bicgstab", tol=1e-10, max_iter=300, precond=ILU0)
    _, st, it, res = O.bicgstab(rp, col, kv, b, tol=1e-10, max_iter=300, precond=ILU0)
    assert out.status == st
    assert abs(out.iterations - it) <= max(3, 0.15 * it)


def test_ilu0_cg_on_the_small_configuration_matches_oracle():
    m = mesh.plain_small(16)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    n = int(l2g.max()) + 1
    s = System(m, l2g)
    rp, col, kv, _, rhs = oracle_system(m, l2g)
    for kind in (0,):
        cfg = _abi.KrylovConfig(1e-10, 5000, ILU0)
        out = _abi.Result()
        x = np.empty(n)
        rc = lib().emg_system_solve(s.h, kind, C.byref(cfg), _abi.ptr(x), 0, None, C.byref(out))
        assert rc == out.status == 0, lib().emg_last_error()
        assert np.linalg.norm(rhs - O.spmv(rp, col, kv, x)) / np.linalg.norm(rhs) <= 2e-10
        xo, _, _, _ = O.pcg(rp, col, kv, rhs, tol=1e-12, max_iter=50000, precond=1)
        assert rel(x, xo) <= 1e-8
    # the mirror of the reference interface takes the same option
    A = api.CsrMatrix(s.matrix(0), owner=s)
    cg = api.CGSolver(api.IterativeSolverConfig(tolerance=1e-10, max_iterations=5000, preconditioner="ILU0"))
    assert cg.get_solver_name() == "CGSolver_ILU0"
    cg.set_matrix(A)
    r = cg.solve(rhs)
    assert r.status == api.SolverStatus.SUCCESS and rel(r.x, xo) <= 1e-8


def test_ilu0_of_a_tridiagonal_matrix_is_exact():
    n = 5000
    i = np.arange(n)
    diag = 4.0 + (i % 5) * 0.3
    rows = np.concatenate([i, i[1:], i[:-1]])
    cols = np.concatenate([i, i[:-1], i[1:]])
    vals = np.concatenate([diag, -np.ones(n - 1), -np.ones(n - 1)])
    order = np.lexsort((cols, rows))
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    A = HostCsr(rp, cols[order].astype(np.int32), vals[order])
    b = np.sin(0.01 * i) + 1.0
    x, out = solve(A.h, b, "cg", tol=1e-12, max_iter=50, precond=ILU0)
    assert out.status == 0 and out.iterations == 1
    xo, _, _, _ = O.pcg(rp.astype(np.int64), cols[order].astype(np.int32), vals[order], b, tol=1e-14,
                        max_iter=10000, precond=0)
    assert rel(x, xo) <= 1e-10


@pytest.mark.parametrize("case", ["zero_pivot", "missing_diagonal"])
def test_ilu0_breakdown_runs_without_preconditioner(case):
    # block diag( [[1, 2], [2, 4 + eps]] ) ... : the second pivot is eps
    n = 400
    rows, cols, vals = [], [], []
    for k in range(0, n, 2):
        a = [[1.0, 2.0], [2.0, 4.0]] if case == "zero_pivot" else [[0.0, 1.0], [1.0, 3.0]]
        for r_ in range(2):
            for c_ in range(2):
                if case == "missing_diagonal" and r_ == c_ == 0:
                    continue
                rows.append(k + r_)
                cols.append(k + c_)
                vals.append(a[r_][c_] + (0.5 if r_ == c_ else 0.0) * (k % 3))
    rows, cols, vals = map(np.asarray, (rows, cols, vals))
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    A = HostCsr(rp, cols.astype(np.int32), vals)
    b = np.linspace(1.0, 2.0, n)
    for kind in ("cg", "bicgstab"):
        x0, o0 = solve(A.h, b, kind, tol=1e-10, max_iter=300, precond=0)
        x2, o2 = solve(A.h, b, kind, tol=1e-10, max_iter=300, precond=ILU0)
        assert (o2.status, o2.iterations) == (o0.status, o0.iterations)
        np.testing.assert_array_equal(np.nan_to_num(x2), np.nan_to_num(x0))
