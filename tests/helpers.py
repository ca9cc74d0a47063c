"""Shared helpers of the GPU parity tests (the product path through the C ABI,
compared with the oracle)."""
import ctypes as C

import numpy as np

from emagddm_b200 import _abi, mesh
from oracle import oracle as O

L = None


def lib():
    global L
    if L is None:
        L = _abi.lib()
    return L


class System:
    """emg_system built from host arrays, assembled with the mesh's materials."""

    def __init__(self, m, l2g, flags=0, sigma=None, n_dofs=0):
        self.m = m
        self.l2g = np.ascontiguousarray(l2g, np.int32)
        xyz = np.ascontiguousarray(m.xyz, np.float64)
        tets = np.ascontiguousarray(m.tets, np.int32)
        mat = np.ascontiguousarray(m.material, np.int32)
        self.h = C.c_void_p()
        et = mesh.TYPE_OF_NODES[tets.shape[1]]
        _abi.check(lib().emg_system_create_typed(et, xyz.shape[0], _abi.ptr(xyz), tets.shape[0], _abi.ptr(tets),
                                                 _abi.ptr(mat), _abi.ptr(self.l2g), n_dofs, 0, None,
                                                 C.byref(self.h)), "emg_system_create_typed")
        self.nu = np.ascontiguousarray(m.nu, np.float64)
        self.sigma = np.ascontiguousarray(m.sigma if sigma is None else sigma, np.float64)
        self.flags = flags
        self.assemble()

    def assemble(self):
        arr, ns = _abi.sources_array(self.m.sources)
        _abi.check(lib().emg_system_assemble(self.h, _abi.ptr(self.nu), _abi.ptr(self.sigma), len(self.nu),
                                             C.cast(arr, C.c_void_p) if arr is not None else None, ns,
                                             self.flags, None), "emg_system_assemble")

    def export(self):
        n, nnz = C.c_int64(), C.c_int64()
        lib().emg_system_info(self.h, C.byref(n), C.byref(nnz))
        rp = np.empty(n.value + 1, np.int32)
        col = np.empty(nnz.value, np.int32)
        kv = np.empty(nnz.value)
        mv = np.empty(nnz.value) if self.flags & _abi.FLAG_MASS else None
        rhs = np.empty(n.value)
        _abi.check(lib().emg_system_export(self.h, _abi.ptr(rp), _abi.ptr(col), _abi.ptr(kv), _abi.ptr(mv),
                                           _abi.ptr(rhs)), "emg_system_export")
        return rp, col, kv, mv, rhs

    def matrix(self, which=0):
        return lib().emg_system_matrix(self.h, which)

    def __del__(self):
        if getattr(self, "h", None):
            lib().emg_system_destroy(self.h)
            self.h = None


def oracle_system(m, l2g, flags=0, sigma=None):
    n = int(np.max(l2g)) + 1
    mm = m
    if sigma is not None:
        mm = mesh.CubeMesh(**{**m.__dict__, "sigma": np.asarray(sigma, np.float64)})
    return O.assemble(mm, l2g, n, flags=flags)


def solve(A, b, kind="cg", tol=1e-8, max_iter=1000, precond=1):
    b = np.ascontiguousarray(b, np.float64)
    x = np.empty_like(b)
    cfg = _abi.KrylovConfig(tol, max_iter, precond)
    out = _abi.Result()
    fn = lib().emg_cg_solve if kind == "cg" else lib().emg_bicgstab_solve
    rc = fn(A, _abi.ptr(b), _abi.ptr(x), C.byref(cfg), C.byref(out))
    assert rc == out.status, (rc, out.status, lib().emg_last_error())
    return x, out


class HostCsr:
    def __init__(self, rp, col, val):
        rp = np.ascontiguousarray(rp, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        self.h = C.c_void_p()
        _abi.check(lib().emg_csr_create(rp.size - 1, _abi.ptr(rp), _abi.ptr(col), _abi.ptr(val), None,
                                        C.byref(self.h)), "emg_csr_create")

    def __del__(self):
        if getattr(self, "h", None):
            lib().emg_csr_destroy(self.h)
            self.h = None
