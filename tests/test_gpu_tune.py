"""The launch-configuration autotuner: the SELL SpMV grid of a matrix, the
batched loop's SpMV grid and the FETI-DP solve kernels' CTA widths are
chosen by timing candidates on the device; the decision table lists every
candidate's median time, the chosen value is one of the candidates, and the
solutions still match the FP64 oracle (1e-8 relative, the solve path's bar).
With tuning switched off the built-in defaults are used."""
import numpy as np
import pytest

from emagddm_b200 import _abi, batch, fetidp, mesh
from oracle import oracle as O
from tests.helpers import System, lib, oracle_system, solve

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _check_family(prefix):
    rep = _abi.tune_report()
    keys = [k for k in rep if k.startswith(prefix + "|")]
    assert keys, (prefix, list(rep))
    for k in keys:
        cands = {int(c) for c in rep[k]["candidates_ms"]}
        assert rep[k]["value"] in cands and len(cands) >= 1
        assert all(v > 0 for v in rep[k]["candidates_ms"].values())
    return rep


def test_spmv_grid_is_tuned_and_the_solve_holds():
    m = mesh.plain_scale(20)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    s = System(m, l2g)
    rp, col, kv, _, rhs = oracle_system(m, l2g)
    x, out = solve(s.matrix(0), rhs, "cg", tol=1e-10, max_iter=20000, precond=1)
    assert out.status == 0
    _check_family("sell.spmv_grid")
    xo, _, _, _ = O.pcg(rp, col, kv, rhs, tol=1e-12, max_iter=50000, precond=1)
    assert rel(x, xo) <= 1e-8


def test_fetidp_solve_kernels_are_tuned():
    m = mesh.plain_scale(12)
    part = mesh.jittered_partition(m, 2)
    fd = fetidp.FetiDP(m, part, 8)
    assert fd.factor() == 0, lib().emg_last_error()
    for fam in ("feti.front_pivot_threads", "feti.front_update_rows", "feti.dense_column_warps"):
        _check_family(fam)
    x, rc, out = fd.solve(tol=1e-11, max_iter=3000)
    assert rc == 0
    rp, col, kv, _, rhs = oracle_system(m, fd.map.l2g)
    xo, st, _, res = O.pcg(rp, col, kv, rhs, tol=1e-13, max_iter=50000, precond=1)
    assert rel(x, xo) <= 1e-8


def test_batch_spmv_grid_is_tuned():
    import torch
    b = batch.build_batch(batch.make_instances(12, nmin=6, nmax=12), threads=2)
    S = batch.BatchSystem(b)
    x = torch.zeros(b.n_rows, dtype=torch.float64, device="cuda")
    rc, res = S.solve(x.data_ptr(), tol=1e-10, max_iter=20000)
    torch.cuda.synchronize()
    assert rc == 0, lib().emg_last_error()
    _check_family("batch.spmv_grid")


def test_tuning_off_keeps_defaults():
    before = _abi.tune_report()
    try:
        _abi.check(lib().emg_tune_enable(0), "emg_tune_enable")
        m = mesh.plain_scale(9)
        l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
        s = System(m, l2g)
        _, _, _, _, rhs = oracle_system(m, l2g)
        _, out = solve(s.matrix(0), rhs, "cg", tol=1e-10, max_iter=20000, precond=1)
        assert out.status == 0
        assert _abi.tune_report().keys() == before.keys()  # nothing timed, nothing recorded
    finally:
        lib().emg_tune_enable(1)
