"""ctypes wrapper of the CPU oracle (emg_oracle.c) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py (CPU baseline / reference
arm) import this module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
I64P = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

STATUS = {0: "SUCCESS", 1: "NUMERICAL_ERROR", 2: "DIVERGED", 3: "MAX_ITER_REACHED", 4: "INVALID_INPUT"}
FLAG_MASS, FLAG_NO_EDGE_SIGNS, FLAG_PIOLA_LITERAL, FLAG_QUAD3_LITERAL = 1, 2, 4, 8
GAUGE_NONE, GAUGE_REF, GAUGE_BOUNDARY_FIRST = -1, 0, 1


class OrcSource(C.Structure):
    _fields_ = [("kind", C.c_int32), ("j", C.c_double * 3), ("p", C.c_double * 6)]


def build() -> str:
    path = os.path.join(_HERE, "libemg_oracle.so")
    src = os.path.join(_HERE, "emg_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "libemg_oracle.so"])
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        L = _LIB
        L.orc_edge_ids.argtypes = [C.c_int64, I32P, I32P, I32P, C.POINTER(C.c_int64)]
        L.orc_dof_build.argtypes = [C.c_int64, I32P, I32P, I32P, C.c_int64, C.c_int64, I32P,
                                    C.c_int32, C.c_int32, I32P, I32P, C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        L.orc_element.argtypes = [F64P, C.c_double, C.c_double, C.c_void_p, C.c_int32, C.c_int32,
                                  F64P, F64P, F64P]
        L.orc_element.restype = None
        L.orc_edge_signs.argtypes = [I32P, I32P]
        L.orc_edge_signs.restype = None
        L.orc_pattern.argtypes = [C.c_int64, I32P, C.c_int64, I64P, C.c_void_p, C.POINTER(C.c_int64)]
        L.orc_assemble.argtypes = [C.c_int64, F64P, C.c_int64, I32P, I32P, I32P, F64P, F64P,
                                   C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int64, I64P,
                                   I32P, F64P, C.c_void_p, C.c_void_p]
        L.orc_spmv.argtypes = [C.c_int64, I64P, I32P, F64P, F64P, F64P]
        L.orc_spmv.restype = None
        for f in (L.orc_pcg, L.orc_bicgstab):
            f.argtypes = [C.c_int64, I64P, I32P, F64P, F64P, F64P, C.c_double, C.c_int32,
                          C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.orc_pcg_snap.argtypes = L.orc_pcg.argtypes + [C.c_double, F64P, C.POINTER(C.c_int32)]
        L.orc_num_threads.restype = C.c_int
        L.orc_edge_ids_typed.argtypes = [C.c_int32, C.c_int64, I32P, I32P, I32P, C.POINTER(C.c_int64)]
        L.orc_dof_build_typed.argtypes = [C.c_int32] + L.orc_dof_build.argtypes
        L.orc_pattern_typed.argtypes = [C.c_int32] + L.orc_pattern.argtypes
        L.orc_assemble_typed.argtypes = [C.c_int32] + L.orc_assemble.argtypes
        for f in (L.orc_hex_basis, L.orc_hex_curl):
            f.argtypes = [C.c_int, F64P, F64P]
            f.restype = None
        L.orc_hex_jacobian.argtypes = [F64P, F64P, F64P, C.POINTER(C.c_double)]
        L.orc_hex_jacobian.restype = None
        L.orc_element_hex.argtypes = L.orc_element.argtypes
        L.orc_element_hex.restype = None
        L.orc_edge_signs_hex.argtypes = [I32P, I32P]
        L.orc_edge_signs_hex.restype = None
        L.orc_shape_circulation.argtypes = [C.c_int32, C.c_int, C.c_int, C.c_int]
        L.orc_shape_circulation.restype = C.c_double
        L.orc_shape_grad_residual.argtypes = [C.c_int32, F64P]
        L.orc_shape_grad_residual.restype = C.c_double
    return _LIB


ELEM_TET4_EDGE, ELEM_HEX8_EDGE, ELEM_PRISM6_EDGE, ELEM_PYRAMID5_EDGE = 0, 1, 2, 3
ELEM_MIXED = 4  # rows of 8 node slots (-1 padded) + the element type; 12 edge slots
_TYPE_OF_NODES = {4: ELEM_TET4_EDGE, 8: ELEM_HEX8_EDGE, 6: ELEM_PRISM6_EDGE, 5: ELEM_PYRAMID5_EDGE, 9: ELEM_MIXED}
_EDGES = {ELEM_TET4_EDGE: 6, ELEM_HEX8_EDGE: 12, ELEM_PRISM6_EDGE: 9, ELEM_PYRAMID5_EDGE: 8, ELEM_MIXED: 12}
_TYPE_OF_EDGES = {v: k for k, v in _EDGES.items()}


def elem_type_of(elems) -> int:
    """Element type of a (T, nodes) array: 4 TET4_EDGE, 8 HEX8_EDGE, 6
    PRISM6_EDGE, 5 PYRAMID5_EDGE, 9 a mixed mesh."""
    return _TYPE_OF_NODES[np.asarray(elems).shape[-1]]


def edges_per_elem(elem_type: int) -> int:
    return _EDGES[elem_type]


def shape_circulation(elem_type, k, e, n=2000):
    """Circulation of PRISM6_EDGE / PYRAMID5_EDGE basis k along edge e."""
    return lib().orc_shape_circulation(elem_type, k, e, n)


def shape_grad_residual(elem_type, x):
    """max |grad N_a - sum_k (N_a(b_k) - N_a(a_k)) W_k| at reference point x."""
    return lib().orc_shape_grad_residual(elem_type, np.ascontiguousarray(x, np.float64))


def sources_array(sources):
    if not sources:
        return None, 0
    arr = (OrcSource * len(sources))()
    for k, s in enumerate(sources):
        arr[k].kind = int(s.kind)
        for i in range(3):
            arr[k].j[i] = float(s.j[i])
        for i in range(6):
            arr[k].p[i] = float(s.p[i])
    return arr, len(sources)


def edge_ids(tets):
    """Edge IDs of (T, 4) tets or (T, 8) hexes: (T, 6|12) element edges and
    the (E, 2) sorted node pairs."""
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    et = elem_type_of(tets)
    T, epe = tets.shape[0], edges_per_elem(et)
    elem_edge = np.empty(epe * T, np.int32)
    edge_nodes = np.empty(2 * epe * T, np.int32)
    ne = C.c_int64()
    rc = lib().orc_edge_ids_typed(et, T, tets.ravel(), elem_edge, edge_nodes, C.byref(ne))
    assert rc == 0, rc
    return elem_edge.reshape(T, epe), edge_nodes[: 2 * ne.value].reshape(-1, 2)


def dof_build(tets, dirichlet, gauge=GAUGE_REF, n_holes=0, elem_edge=None, edge_nodes=None):
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    et = elem_type_of(tets)
    epe = edges_per_elem(et)
    if elem_edge is None:
        elem_edge, edge_nodes = edge_ids(tets)
    T, E = tets.shape[0], edge_nodes.shape[0]
    d = np.ascontiguousarray(dirichlet, dtype=np.int32).reshape(-1)
    l2g = np.empty(epe * T, np.int32)
    edge_dof = np.empty(E, np.int32)
    nf, nd, root = C.c_int64(), C.c_int64(), C.c_int32()
    rc = lib().orc_dof_build_typed(et, T, tets.ravel(), np.ascontiguousarray(elem_edge, np.int32).ravel(),
                                   np.ascontiguousarray(edge_nodes, np.int32).ravel(), E, d.size // 2,
                                   d if d.size else np.zeros(2, np.int32), n_holes, gauge, l2g, edge_dof,
                                   C.byref(nf), C.byref(nd), C.byref(root))
    assert rc == 0, rc
    return dict(elem_edge=elem_edge, edge_nodes=edge_nodes, l2g=l2g.reshape(T, epe),
                edge_dof=edge_dof, n_edges=E, n_free=nf.value, n_dofs=nd.value, root=root.value)


def dof_build_av(elems, dof_type, dirichlet, scalar_dirichlet, gauge=GAUGE_REF, n_holes=0, n_nodes=None):
    """EMDOFManager with per-element DOFType (0 SCALAR_ONLY, 1 VECTOR_EDGE_ONLY,
    2 MIXED_AV): rows of npe + epe entries (Local2Global::indices, padded -2)."""
    elems = np.ascontiguousarray(elems, dtype=np.int32)
    et = elem_type_of(elems)
    w = elems.shape[1] + edges_per_elem(et)
    T = elems.shape[0]
    if n_nodes is None:
        n_nodes = int(elems.max()) + 1 if elems.size else 0
    dt = np.ascontiguousarray(dof_type, np.int32)
    d = np.ascontiguousarray(dirichlet, dtype=np.int32).reshape(-1)
    sd = np.ascontiguousarray(scalar_dirichlet, dtype=np.int32).reshape(-1)
    l2g = np.empty(w * T, np.int32)
    nsf, nf, nd = C.c_int64(), C.c_int64(), C.c_int64()
    L = lib()
    L.orc_dof_build_av.argtypes = [C.c_int32, C.c_int64, C.c_int64, I32P, I32P, C.c_int64, I32P, C.c_int64, I32P,
                                   C.c_int32, C.c_int32, I32P, C.c_void_p, C.c_void_p, C.c_void_p]
    rc = L.orc_dof_build_av(et, n_nodes, T, elems.ravel(), dt, d.size // 2, d if d.size else np.zeros(2, np.int32),
                            sd.size, sd if sd.size else np.zeros(1, np.int32), n_holes, gauge, l2g,
                            C.byref(nsf), C.byref(nf), C.byref(nd))
    assert rc == 0, rc
    return dict(l2g=l2g.reshape(T, w), n_scalar_free=nsf.value, n_free=nf.value, n_dofs=nd.value)


def element(X, nu=1.0, sigma=0.0, sources=(), flags=0):
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(12)
    K, M, F = np.empty(36), np.empty(36), np.empty(6)
    arr, ns = sources_array(list(sources))
    lib().orc_element(X, nu, sigma, C.cast(arr, C.c_void_p) if arr is not None else None, ns,
                      flags, K, M, F)
    return K.reshape(6, 6), M.reshape(6, 6), F


def edge_signs(tet):
    if len(tet) == 8:
        s = np.empty(12, np.int32)
        lib().orc_edge_signs_hex(np.ascontiguousarray(tet, np.int32), s)
        return s
    s = np.empty(6, np.int32)
    lib().orc_edge_signs(np.ascontiguousarray(tet, np.int32), s)
    return s


def element_hex(X, nu=1.0, sigma=0.0, sources=(), flags=0):
    """HEX8_EDGE element matrices (12 x 12 K, M; F 12) of the 8 nodes X."""
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(24)
    K, M, F = np.empty(144), np.empty(144), np.empty(12)
    arr, ns = sources_array(list(sources))
    lib().orc_element_hex(X, nu, sigma, C.cast(arr, C.c_void_p) if arr is not None else None, ns,
                          flags, K, M, F)
    return K.reshape(12, 12), M.reshape(12, 12), F


def hex_basis(x):
    """(12, 3) reference values and (12, 3) reference curls at x."""
    x = np.ascontiguousarray(x, np.float64)
    W, Cu = np.empty((12, 3)), np.empty((12, 3))
    for k in range(12):
        w, c = np.empty(3), np.empty(3)
        lib().orc_hex_basis(k, x, w)
        lib().orc_hex_curl(k, x, c)
        W[k], Cu[k] = w, c
    return W, Cu


def hex_jacobian(X, x):
    J = np.empty(9)
    det = C.c_double()
    lib().orc_hex_jacobian(np.ascontiguousarray(X, np.float64).reshape(24), np.ascontiguousarray(x, np.float64),
                           J, C.byref(det))
    return J.reshape(3, 3), det.value


def pattern(l2g, n):
    """Merged CSR pattern; l2g is (T, 6) for tets or (T, 12) for hexes (a flat
    array is read as tets)."""
    l2g = np.asarray(l2g)
    et = _TYPE_OF_EDGES[l2g.shape[1]] if l2g.ndim == 2 else ELEM_TET4_EDGE
    l2g = np.ascontiguousarray(l2g, dtype=np.int32).ravel()
    T = l2g.size // edges_per_elem(et)
    rp = np.empty(n + 1, np.int64)
    nnz = C.c_int64()
    rc = lib().orc_pattern_typed(et, T, l2g, n, rp, None, C.byref(nnz))
    assert rc == 0, rc
    col = np.empty(max(nnz.value, 1), np.int32)
    rc = lib().orc_pattern_typed(et, T, l2g, n, rp, col.ctypes.data_as(C.c_void_p), C.byref(nnz))
    assert rc == 0, rc
    return rp, col[: nnz.value]


def assemble(mesh, l2g, n, flags=0, rp=None, col=None):
    """Merged CSR (int64 row_ptr, int32 col), K values, M values, rhs."""
    et = elem_type_of(mesh.tets)
    if rp is None:
        rp, col = pattern(np.asarray(l2g).reshape(mesh.n_tets, edges_per_elem(et)), n)
    nnz = int(rp[-1])
    kval = np.empty(nnz)
    mval = np.empty(nnz) if flags & FLAG_MASS else None
    rhs = np.empty(n)
    arr, ns = sources_array(mesh.sources)
    rc = lib().orc_assemble_typed(et, mesh.n_nodes, np.ascontiguousarray(mesh.xyz).ravel(), mesh.n_tets,
                            np.ascontiguousarray(mesh.tets, np.int32).ravel(),
                            np.ascontiguousarray(mesh.material, np.int32),
                            np.ascontiguousarray(l2g, np.int32).ravel(),
                            np.ascontiguousarray(mesh.nu, np.float64),
                            np.ascontiguousarray(mesh.sigma, np.float64), len(mesh.nu),
                            C.cast(arr, C.c_void_p) if arr is not None else None, ns, flags, n,
                            rp, col, kval,
                            mval.ctypes.data_as(C.c_void_p) if mval is not None else None,
                            rhs.ctypes.data_as(C.c_void_p))
    assert rc == 0, rc
    return rp, col, kval, mval, rhs


def spmv(rp, col, val, x):
    y = np.empty(rp.size - 1)
    lib().orc_spmv(rp.size - 1, rp, col, val, np.ascontiguousarray(x, np.float64), y)
    return y


def _krylov(fn, rp, col, val, b, tol, max_iter, precond):
    n = rp.size - 1
    x = np.empty(n)
    it, res = C.c_int32(), C.c_double()
    st = fn(n, rp, col, val, np.ascontiguousarray(b, np.float64), x, tol, max_iter, precond,
            C.byref(it), C.byref(res))
    return x, st, it.value, res.value


def pcg(rp, col, val, b, tol=1e-8, max_iter=1000, precond=1):
    return _krylov(lib().orc_pcg, rp, col, val, b, tol, max_iter, precond)


def pcg_snap(rp, col, val, b, tol=1e-12, snap_tol=1e-8, max_iter=1000, precond=1):
    """pcg to `tol` that also returns the iterate at which a solve to
    `snap_tol` stops: (x, status, iterations, residual, x_snap, snap_iter)."""
    n = rp.size - 1
    x, xs = np.empty(n), np.empty(n)
    it, res, sit = C.c_int32(), C.c_double(), C.c_int32()
    st = lib().orc_pcg_snap(n, rp, col, val, np.ascontiguousarray(b, np.float64), x, tol, max_iter, precond,
                            C.byref(it), C.byref(res), snap_tol, xs, C.byref(sit))
    return x, st, it.value, res.value, xs, sit.value


def bicgstab(rp, col, val, b, tol=1e-8, max_iter=1000, precond=1):
    return _krylov(lib().orc_bicgstab, rp, col, val, b, tol, max_iter, precond)


def num_threads() -> int:
    return int(lib().orc_num_threads())
