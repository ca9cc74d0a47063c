"""Batched many-instance solves: the union of disjoint instance meshes is one
block-diagonal system solved in lockstep (emg_batch_cg_solve_device).
Each block must match the oracle's solve of that instance alone:
solutions to 1e-8 relative, matrices to 1e-12 of their scale."""
import ctypes as C

import numpy as np
import pytest

from emagddm_b200 import _abi, batch, mesh
from oracle import oracle as O

CASES = [(3, 1), (5, 2), (4, 3), (6, 4), (2, 5), (7, 6), (3, 7)]


def instances():
    return [mesh.random_instance(n, s) for n, s in CASES]


def test_batch_layout_cpu():
    b = batch.build_batch(instances(), threads=2)
    assert b.block_row_ptr[0] == 0 and len(b.block_row_ptr) == len(CASES) + 1
    for k, (m, l) in enumerate(zip(b.instances, b.l2g_each)):
        o = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
        np.testing.assert_array_equal(l, o["l2g"])
        assert b.block_row_ptr[k + 1] - b.block_row_ptr[k] == int(o["l2g"].max()) + 1
    assert b.l2g.max() + 1 == b.n_rows
    assert len(b.sources) == len(CASES) and b.tet_source.max() == len(CASES) - 1
    assert b.material.max() == len(b.nu) - 1
    sizes = batch.instance_sizes(512)
    assert min(sizes) >= 8 and max(sizes) <= 32 and len(set(sizes)) > 10


@pytest.mark.gpu
def test_batch_blocks_match_oracle():
    import torch
    b = batch.build_batch(instances(), threads=2)
    S = batch.BatchSystem(b)
    rp, col, kv, rhs = S.export()
    x = torch.zeros(b.n_rows, dtype=torch.float64, device="cuda")
    rc, res = S.solve(x.data_ptr(), tol=1e-12, max_iter=20000)
    torch.cuda.synchronize()
    assert rc == _abi.EMG_SUCCESS, (rc, res, _abi.lib().emg_last_error())
    xs = x.cpu().numpy()
    for k, m in enumerate(b.instances):
        r0, r1 = b.block_row_ptr[k], b.block_row_ptr[k + 1]
        l2g = b.l2g_each[k]
        orp, ocol, okv, _, orhs = O.assemble(m, l2g, r1 - r0)
        # the block of the batched matrix equals the instance's own matrix
        blk = slice(rp[r0], rp[r1])
        np.testing.assert_array_equal(rp[r0:r1 + 1] - rp[r0], orp)
        np.testing.assert_array_equal(col[blk] - r0, ocol)
        assert np.abs(kv[blk] - okv).max() <= 1e-12 * np.abs(okv).max()
        assert np.abs(rhs[r0:r1] - orhs).max() <= 1e-12 * max(np.abs(orhs).max(), 1e-300)
        xo, st, it, _ = O.pcg(orp, ocol, okv, orhs, tol=1e-12, max_iter=20000, precond=1)
        assert res[k]["status"] == st == 0
        assert abs(res[k]["iterations"] - it) <= max(3, 0.15 * it)
        assert np.linalg.norm(xs[r0:r1] - xo) <= 1e-8 * max(np.linalg.norm(xo), 1e-300)


@pytest.mark.gpu
def test_batch_statuses_and_coupling_check():
    import torch
    b = batch.build_batch(instances()[:3], threads=2)
    S = batch.BatchSystem(b)
    x = torch.zeros(b.n_rows, dtype=torch.float64, device="cuda")
    rc, res = S.solve(x.data_ptr(), tol=1e-14, max_iter=4)
    assert rc == _abi.EMG_MAX_ITER_REACHED
    assert all(r["status"] == _abi.EMG_MAX_ITER_REACHED and r["iterations"] == 4 for r in res)
    # a partition that cuts through a block couples two "systems": rejected
    L = _abi.lib()
    bad = b.block_row_ptr.copy()
    bad[1] += 1
    out = (_abi.Result * 3)()
    cfg = _abi.KrylovConfig(1e-8, 100, 1)
    rc = L.emg_batch_cg_solve_device(L.emg_system_matrix(S.h, 0), 3, _abi.ptr(bad),
                                     C.c_void_p(L.emg_system_rhs_device(S.h)), C.c_void_p(x.data_ptr()),
                                     C.byref(cfg), None, out)
    assert rc == _abi.EMG_INVALID_INPUT
    assert b"couples" in L.emg_last_error()


@pytest.mark.gpu
def test_batch_zero_block_rhs_finishes_at_once():
    """A block whose right-hand side is zero finishes in the first list
    (SUCCESS, 0 iterations, x = 0) while the others iterate to the oracle's
    solutions; blocks leave the active list as they converge."""
    import torch
    b = batch.build_batch(instances(), threads=2)
    S = batch.BatchSystem(b)
    rp, col, kv, rhs = S.export()
    r0, r1 = b.block_row_ptr[2], b.block_row_ptr[3]
    rhs = rhs.copy()
    rhs[r0:r1] = 0.0
    bd = torch.from_numpy(rhs).cuda()
    x = torch.full((b.n_rows,), 7.0, dtype=torch.float64, device="cuda")
    L = _abi.lib()
    nb = len(b.instances)
    out = (_abi.Result * nb)()
    cfg = _abi.KrylovConfig(1e-10, 20000, 1)
    rc = L.emg_batch_cg_solve_device(L.emg_system_matrix(S.h, 0), nb, _abi.ptr(b.block_row_ptr),
                                     C.c_void_p(bd.data_ptr()), C.c_void_p(x.data_ptr()), C.byref(cfg), None, out)
    torch.cuda.synchronize()
    assert rc == _abi.EMG_SUCCESS, L.emg_last_error()
    xs = x.cpu().numpy()
    assert out[2].status == _abi.EMG_SUCCESS and out[2].iterations == 0
    assert np.all(xs[r0:r1] == 0.0)
    its = []
    for k in range(nb):
        if k == 2:
            continue
        a0, a1 = b.block_row_ptr[k], b.block_row_ptr[k + 1]
        blk = slice(rp[a0], rp[a1])
        orp = (rp[a0:a1 + 1] - rp[a0]).astype(np.int64)
        ocol = (col[blk] - a0).astype(np.int32)
        xo, st, it, _ = O.pcg(orp, ocol, kv[blk], rhs[a0:a1], tol=1e-10, max_iter=20000, precond=1)
        assert out[k].status == st == 0
        assert abs(out[k].iterations - it) <= max(3, 0.15 * it)
        assert np.linalg.norm(xs[a0:a1] - xo) <= 1e-8 * np.linalg.norm(xo)
        its.append(out[k].iterations)
    assert len(set(its)) > 3  # blocks finish at different iterations


@pytest.mark.gpu
def test_batch_more_blocks_than_one_list_chunk():
    """1,100 small blocks: the active list is built in chunks of 1,024 blocks;
    every block converges and a sample matches the oracle's own solves."""
    import torch
    inst = [mesh.random_instance(2 + (k % 3), 1000 + k) for k in range(1100)]
    b = batch.build_batch(inst, threads=4)
    S = batch.BatchSystem(b)
    rp, col, kv, rhs = S.export()
    x = torch.zeros(b.n_rows, dtype=torch.float64, device="cuda")
    rc, res = S.solve(x.data_ptr(), tol=1e-10, max_iter=5000)
    torch.cuda.synchronize()
    assert rc == _abi.EMG_SUCCESS, (rc, _abi.lib().emg_last_error())
    assert all(r["status"] == _abi.EMG_SUCCESS for r in res)
    xs = x.cpu().numpy()
    for k in (0, 511, 1023, 1024, 1099):
        a0, a1 = b.block_row_ptr[k], b.block_row_ptr[k + 1]
        blk = slice(rp[a0], rp[a1])
        orp = (rp[a0:a1 + 1] - rp[a0]).astype(np.int64)
        ocol = (col[blk] - a0).astype(np.int32)
        xo, st, it, _ = O.pcg(orp, ocol, kv[blk], rhs[a0:a1], tol=1e-10, max_iter=5000, precond=1)
        assert st == 0 and abs(res[k]["iterations"] - it) <= max(3, 0.15 * it)
        assert np.linalg.norm(xs[a0:a1] - xo) <= 1e-8 * max(np.linalg.norm(xo), 1e-300)


@pytest.mark.gpu
def test_batch_with_empty_blocks():
    """Instances without free DOFs (n = 1 cubes, every edge on the boundary)
    give empty blocks, two of them adjacent: they finish at once and the
    blocks around them still match the oracle."""
    import torch
    inst = [mesh.random_instance(3, 1), mesh.random_instance(1, 2), mesh.random_instance(1, 3),
            mesh.random_instance(4, 4), mesh.random_instance(1, 5)]
    b = batch.build_batch(inst, threads=2)
    assert b.block_row_ptr[1] == b.block_row_ptr[3] and b.block_row_ptr[4] == b.block_row_ptr[5]
    S = batch.BatchSystem(b)
    rp, col, kv, rhs = S.export()
    x = torch.zeros(b.n_rows, dtype=torch.float64, device="cuda")
    rc, res = S.solve(x.data_ptr(), tol=1e-10, max_iter=5000)
    torch.cuda.synchronize()
    assert rc == _abi.EMG_SUCCESS, (rc, _abi.lib().emg_last_error())
    for k in (1, 2, 4):
        assert res[k]["status"] == _abi.EMG_SUCCESS and res[k]["iterations"] == 0
    xs = x.cpu().numpy()
    for k in (0, 3):
        a0, a1 = b.block_row_ptr[k], b.block_row_ptr[k + 1]
        blk = slice(rp[a0], rp[a1])
        orp = (rp[a0:a1 + 1] - rp[a0]).astype(np.int64)
        ocol = (col[blk] - a0).astype(np.int32)
        xo, st, it, _ = O.pcg(orp, ocol, kv[blk], rhs[a0:a1], tol=1e-10, max_iter=5000, precond=1)
        assert res[k]["status"] == st == 0 and abs(res[k]["iterations"] - it) <= max(3, 0.15 * it)
        assert np.linalg.norm(xs[a0:a1] - xo) <= 1e-8 * np.linalg.norm(xo)
