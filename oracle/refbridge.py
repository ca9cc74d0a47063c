"""ctypes wrapper of oracle/_ref/libemg_ref.so -- TEST INFRASTRUCTURE.

The library is the reference's own C++ sources compiled in place by
oracle/Makefile.ref plus ref_bridge.cpp.  It is built here (where the
reference sources exist) and travels with the repository snapshot; when it is
absent, callers skip the reference comparisons.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(_HERE, "_ref", "libemg_ref.so")
_LIB = None

I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
I64P = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def available() -> bool:
    return os.path.exists(PATH)


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(PATH)
        L = _LIB
        L.refb_quiet.argtypes = [C.c_int]
        L.refb_quiet.restype = None
        L.refb_dof_build.argtypes = [C.c_int64, C.c_int64, I32P, C.c_int64, I32P, C.c_int32,
                                     C.c_int32, I32P, I32P, C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.refb_pattern.argtypes = [C.c_int64, F64P, C.c_int64, I32P, I32P, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int64)]
        L.refb_krylov.argtypes = [C.c_int32, C.c_int64, I64P, I32P, F64P, F64P, F64P, C.c_double,
                                  C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                  C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]
        L.refb_nedelec_tet4.argtypes = [C.c_double, C.c_double, C.c_double, F64P, F64P]
        L.refb_nedelec_tet4.restype = None
        L.refb_quadrature.argtypes = [C.c_int32, C.c_int32, F64P]
        L.refb_integrator_k.argtypes = [F64P, C.c_double, F64P]
        L.refb_dof_build_typed.argtypes = [C.c_int32] + L.refb_dof_build.argtypes
        L.refb_pattern_typed.argtypes = [C.c_int32] + L.refb_pattern.argtypes
        L.refb_nedelec_hex8.argtypes = [C.c_double, C.c_double, C.c_double, F64P, F64P]
        L.refb_nedelec_hex8.restype = None
        L.refb_hex8_jacobian.argtypes = [F64P, C.c_double, C.c_double, C.c_double, F64P, C.POINTER(C.c_double)]
        L.refb_quadrature_hex.argtypes = [C.c_int32, C.c_int32, F64P]
        L.refb_integrator_k_hex.argtypes = [F64P, C.c_double, F64P]
        L.refb_quiet(1)
    return _LIB


def _elem_type(tets) -> int:
    return {4: 0, 8: 1, 6: 2, 5: 3, 9: 4}[np.asarray(tets).shape[1]]


def dof_build(n_nodes, tets, dirichlet, gauge=True, n_holes=0):
    """GlobalEdgeIDGenerator + EMDOFManager on (T, 4) TET4_EDGE or (T, 8)
    HEX8_EDGE elements."""
    tets = np.ascontiguousarray(tets, np.int32)
    et = _elem_type(tets)
    epe = {0: 6, 1: 12, 2: 9, 3: 8, 4: 12}[et]
    T = tets.shape[0]
    d = np.ascontiguousarray(dirichlet, np.int32).reshape(-1)
    ee = np.empty(epe * T, np.int32)
    l2g = np.empty(epe * T, np.int32)
    ne, nf, nd = C.c_int64(), C.c_int64(), C.c_int64()
    rc = lib().refb_dof_build_typed(et, n_nodes, T, tets.ravel(), d.size // 2,
                                    d if d.size else np.zeros(2, np.int32), n_holes, int(gauge), ee,
                                    l2g, C.byref(ne), C.byref(nf), C.byref(nd))
    assert rc == 0, rc
    return dict(elem_edge=ee.reshape(T, epe), l2g=l2g.reshape(T, epe), n_edges=ne.value,
                n_free=nf.value, n_dofs=nd.value)


def dof_build_av(n_nodes, elems, dof_type, dirichlet, scalar_dirichlet, gauge=True, n_holes=0):
    """EMDOFManager with per-element DOFType (0 SCALAR_ONLY, 1 VECTOR_EDGE_ONLY,
    2 MIXED_AV) and a scalar DIRICHLET marker on `scalar_dirichlet` nodes.
    Rows of l2g: npe + epe entries, Local2Global::indices padded with -2."""
    elems = np.ascontiguousarray(elems, np.int32)
    et = _elem_type(elems)
    w = (8 + 12) if et else (4 + 6)
    T = elems.shape[0]
    dt = np.ascontiguousarray(dof_type, np.int32)
    d = np.ascontiguousarray(dirichlet, np.int32).reshape(-1)
    sd = np.ascontiguousarray(scalar_dirichlet, np.int32).reshape(-1)
    l2g = np.empty(w * T, np.int32)
    nf, nd = C.c_int64(), C.c_int64()
    L = lib()
    L.refb_dof_build_av.argtypes = [C.c_int32, C.c_int64, C.c_int64, I32P, I32P, C.c_int64, I32P, C.c_int64,
                                    I32P, C.c_int32, C.c_int32, I32P, C.c_void_p, C.c_void_p]
    rc = L.refb_dof_build_av(et, n_nodes, T, elems.ravel(), dt, d.size // 2, d if d.size else np.zeros(2, np.int32),
                             sd.size, sd if sd.size else np.zeros(1, np.int32), n_holes, int(gauge), l2g,
                             C.byref(nf), C.byref(nd))
    assert rc == 0, rc
    return dict(l2g=l2g.reshape(T, w), n_free=nf.value, n_dofs=nd.value)


def pattern(xyz, tets, l2g):
    tets = np.ascontiguousarray(tets, np.int32)
    et = _elem_type(tets)
    l2g = np.ascontiguousarray(l2g, np.int32).ravel()
    xyz = np.ascontiguousarray(xyz, np.float64).ravel()
    nnz, raw, nr = C.c_int64(), C.c_int64(), C.c_int64()
    rc = lib().refb_pattern_typed(et, xyz.size // 3, xyz, tets.shape[0], tets.ravel(), l2g, None, None,
                                  C.byref(nnz), C.byref(raw), C.byref(nr))
    assert rc == 0, rc
    rp = np.empty(nr.value + 1, np.int64)
    col = np.empty(nnz.value, np.int32)
    rc = lib().refb_pattern_typed(et, xyz.size // 3, xyz, tets.shape[0], tets.ravel(), l2g,
                                  rp.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                                  C.byref(nnz), C.byref(raw), C.byref(nr))
    assert rc == 0, rc
    return rp, col, raw.value


def krylov(kind, rp, col, val, b, tol=1e-8, max_iter=1000, precond=1):
    """kind 0 = CGSolver, 1 = BiCGSTABSolver.  Returns x, status, iterations,
    relative residual, set_matrix ms, solve ms."""
    n = rp.size - 1
    x = np.zeros(n)
    it, res, s_ms, t_ms = C.c_int32(), C.c_double(), C.c_double(), C.c_double()
    st = lib().refb_krylov(kind, n, np.ascontiguousarray(rp, np.int64),
                           np.ascontiguousarray(col, np.int32), np.ascontiguousarray(val, np.float64),
                           np.ascontiguousarray(b, np.float64), x, tol, max_iter, precond,
                           C.byref(it), C.byref(res), C.byref(s_ms), C.byref(t_ms))
    return x, st, it.value, res.value, s_ms.value, t_ms.value


def nedelec_tet4(xi, eta, zeta):
    w, c = np.empty(18), np.empty(18)
    lib().refb_nedelec_tet4(xi, eta, zeta, w, c)
    return w.reshape(6, 3), c.reshape(6, 3)


def quadrature(edge_type, order):
    p = np.zeros(16)
    n = lib().refb_quadrature(edge_type, order, p)
    return p.reshape(4, 4)[:n]


def integrator_k(X, mu=1.0):
    K = np.empty(36)
    rc = lib().refb_integrator_k(np.ascontiguousarray(X, np.float64).ravel(), mu, K)
    assert rc == 0, rc
    return K.reshape(6, 6)


def nedelec_hex8(xi, eta, zeta):
    """evalEdgeFunction / evalCurlEdge of HEX8_EDGE: (12, 3) values, (12, 3) curls."""
    w, c = np.empty(36), np.empty(36)
    lib().refb_nedelec_hex8(xi, eta, zeta, w, c)
    return w.reshape(12, 3), c.reshape(12, 3)


def hex8_jacobian(X, xi, eta, zeta):
    """HEX8 Lagrange calcJacobian of the 8 nodes X: (3, 3) J, det J."""
    J = np.empty(9)
    det = C.c_double()
    rc = lib().refb_hex8_jacobian(np.ascontiguousarray(X, np.float64).ravel(), xi, eta, zeta, J, C.byref(det))
    assert rc == 0, rc
    return J.reshape(3, 3), det.value


def quadrature_hex(edge_type, order):
    p = np.zeros(32)
    n = lib().refb_quadrature_hex(edge_type, order, p)
    return p.reshape(8, 4)[:n]


def integrator_k_hex(X, mu=1.0):
    K = np.empty(144)
    rc = lib().refb_integrator_k_hex(np.ascontiguousarray(X, np.float64).ravel(), mu, K)
    assert rc == 0, rc
    return K.reshape(12, 12)
