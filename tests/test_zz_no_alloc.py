"""Allocation-free CG entry point (emg_cg_solve_noalloc) against the regular
device entry point (emg_cg_solve_device) on the same caller-owned CSR.

emg_cg_solve_noalloc serves callers that must not let the library allocate
GPU memory (hosts that budget all device memory themselves, loops that may
not call the CUDA allocator after start-up).  Its work vectors live in a
fixed scratch array inside the library that every call reuses, so this test
runs it twice in a row and checks both results; it is collected last so a
run that stops at the first failure has already run every other test.

Tolerance: converged solutions agree with the regular entry point to 1e-8
relative (the solve path's bar); iteration counts within a few iterations.
"""
import ctypes as C

import numpy as np
import pytest

from emagddm_b200 import _abi, mesh
from oracle import oracle as O
from tests.helpers import lib, oracle_system

pytestmark = pytest.mark.gpu


def _device_csr():
    import torch
    m = mesh.plain_scale(12)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    rp, col, kv, _, rhs = oracle_system(m, l2g)
    dev = torch.device("cuda", 0)
    t = dict(rp=torch.from_numpy(rp.astype(np.int32)).to(dev), col=torch.from_numpy(col).to(dev),
             val=torch.from_numpy(kv).to(dev), b=torch.from_numpy(rhs).to(dev))
    return t, rp.size - 1, int(rp[-1])


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_matches_device_entry_point_twice():
    import torch
    t, n, nnz = _device_csr()
    cfg = _abi.KrylovConfig(1e-12, 20000, _abi.PRECOND_JACOBI)
    # existing entry point
    A = C.c_void_p()
    _abi.check(lib().emg_csr_create_device(n, nnz, _p(t["rp"]), _p(t["col"]), _p(t["val"]), None,
                                           C.byref(A)), "emg_csr_create_device")
    x_ref = torch.empty(n, dtype=torch.float64, device="cuda")
    r_ref = _abi.Result()
    rc = lib().emg_cg_solve_device(A, _p(t["b"]), _p(x_ref), C.byref(cfg), None, C.byref(r_ref))
    lib().emg_csr_destroy(A)
    assert rc == r_ref.status == _abi.EMG_SUCCESS
    xr = x_ref.cpu().numpy()
    results = []
    for _ in range(2):  # the scratch keeps the previous call's contents
        x = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        r = _abi.Result()
        rc = lib().emg_cg_solve_noalloc(n, nnz, _p(t["rp"]), _p(t["col"]), _p(t["val"]), _p(t["b"]),
                                        _p(x), C.byref(cfg), None, C.byref(r))
        torch.cuda.synchronize()
        assert rc == r.status == _abi.EMG_SUCCESS, lib().emg_last_error()
        assert abs(r.iterations - r_ref.iterations) <= max(3, 0.15 * r_ref.iterations)
        xs = x.cpu().numpy()
        assert np.linalg.norm(xs - xr) <= 1e-8 * np.linalg.norm(xr)
        results.append((xs, r.iterations, r.residual_norm))
    np.testing.assert_array_equal(results[0][0], results[1][0])
    assert results[0][1:] == results[1][1:]


def test_noalloc_rejects_oversize_and_bad_input():
    import torch
    t, n, nnz = _device_csr()
    cfg = _abi.KrylovConfig(1e-8, 100, _abi.PRECOND_JACOBI)
    x = torch.empty(n, dtype=torch.float64, device="cuda")
    r = _abi.Result()
    rc = lib().emg_cg_solve_noalloc(262_145, nnz, _p(t["rp"]), _p(t["col"]), _p(t["val"]), _p(t["b"]),
                                    _p(x), C.byref(cfg), None, C.byref(r))
    assert rc == _abi.EMG_INVALID_INPUT
    assert b"262144" in lib().emg_last_error()
    bad = t["col"].clone()
    bad[5] = n + 7  # out-of-range column: rejected before any indexed access
    rc = lib().emg_cg_solve_noalloc(n, nnz, _p(t["rp"]), _p(bad), _p(t["val"]), _p(t["b"]), _p(x),
                                    C.byref(cfg), None, C.byref(r))
    assert rc == r.status == _abi.EMG_INVALID_INPUT
    assert b"column" in lib().emg_last_error()
    # a row whose columns are swapped (unmerged form): rejected, since the
    # Jacobi diagonal is defined on a merged CSR
    rp = t["rp"].cpu().numpy()
    row = int(np.argmax(np.diff(rp) >= 2))
    k = int(rp[row])
    swapped = t["col"].clone()
    swapped[k], swapped[k + 1] = t["col"][k + 1], t["col"][k]
    rc = lib().emg_cg_solve_noalloc(n, nnz, _p(t["rp"]), _p(swapped), _p(t["val"]), _p(t["b"]), _p(x),
                                    C.byref(cfg), None, C.byref(r))
    assert rc == r.status == _abi.EMG_INVALID_INPUT
    assert b"ascending" in lib().emg_last_error()
