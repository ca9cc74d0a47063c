"""FETI-DP solve of the gauged TET4_EDGE / HEX8_EDGE curl-curl system on one GPU.

The reference declares FETI-DP (``include/fetidp/fetidp_context.hpp:20-66``,
``src/fetidp/fetidp_context.cpp:15-45``: a subdomain count and zeroed
``SubdomainData`` records) but has no operators; this module is the host
mirror of the library's FETI-DP entry points (``emg_dof_build_partitioned``,
``emg_fetidp_*`` in ``include/emagddm_b200.h``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi, mesh
from ._abi import check, lib, ptr


@dataclass
class PartitionedMap:
    """Result of the partitioned tree-cotree gauge."""
    l2g: np.ndarray          # (T, 6 or 12) int32, -1 = Dirichlet or tree edge
    edge_dof: np.ndarray     # (E,) int32
    n_free: int
    n_dofs: int
    n_parts: int
    primal: np.ndarray       # (n_dofs,) int32 flags
    n_primal_fix: int


class _MeshHandle:
    def __init__(self, m):
        self.xyz = np.ascontiguousarray(m.xyz, np.float64)
        self.tets = np.ascontiguousarray(m.tets, np.int32)
        self.material = np.ascontiguousarray(m.material, np.int32)
        d = np.ascontiguousarray(m.dirichlet, np.int32)
        self.h = C.c_void_p()
        et = mesh.TYPE_OF_NODES[self.tets.shape[1]]
        check(lib().emg_mesh_create_typed(et, self.xyz.shape[0], ptr(self.xyz), self.tets.shape[0],
                                          ptr(self.tets), ptr(self.material), d.shape[0], ptr(d) if d.size else None,
                                          0, C.byref(self.h)), "emg_mesh_create_typed")

    def __del__(self, _abi=_abi):
        if getattr(self, "h", None) and _abi._LIB is not None:
            _abi._LIB.emg_mesh_destroy(self.h)
            self.h = None


class _MapHandle:
    def __init__(self, h):
        self.h = h

    def __del__(self, _abi=_abi):
        if getattr(self, "h", None) and _abi._LIB is not None:
            _abi._LIB.emg_dofmap_destroy(self.h)
            self.h = None


def partitioned_dofmap(m, tet_part, n_parts: int, keep_handles: bool = False):
    """Gauge the mesh for a partition; with keep_handles also return the
    (mesh, dofmap) handle owners the FETI-DP solver is created from."""
    mh = _MeshHandle(m)
    part = np.ascontiguousarray(tet_part, np.int32)
    h = C.c_void_p()
    check(lib().emg_dof_build_partitioned(mh.h, ptr(part), int(n_parts), C.byref(h)),
          "emg_dof_build_partitioned")
    ne, nf, nd = C.c_int64(), C.c_int64(), C.c_int64()
    lib().emg_dofmap_info(h, C.byref(ne), C.byref(nf), C.byref(nd))
    l2g = np.empty((m.n_tets, mesh.EDGES_OF_TYPE[m.elem_type]), np.int32)
    ed = np.empty(ne.value, np.int32)
    lib().emg_dofmap_export(h, ptr(l2g), ptr(ed))
    npart, npri, nfix = C.c_int32(), C.c_int64(), C.c_int64()
    pri = np.empty(nd.value, np.int32)
    check(lib().emg_dofmap_partition_info(h, C.byref(npart), C.byref(npri), C.byref(nfix), ptr(pri)),
          "emg_dofmap_partition_info")
    pm = PartitionedMap(l2g, ed, nf.value, nd.value, npart.value, pri, nfix.value)
    if keep_handles:
        return pm, mh, _MapHandle(h)
    lib().emg_dofmap_destroy(h)
    return pm


INFO_KEYS = ("n_parts", "n_dofs", "n_union", "n_lambda", "n_coarse", "n_fronts", "n_levels", "max_front",
             "max_pivots", "factor_doubles", "update_pool_doubles", "dual_block_doubles", "sum_nI", "sum_nD",
             "sum_nP", "max_nD", "max_children", "flops_panel", "flops_update", "flops_dense",
             "sym_tile_doubles", "face_block_doubles")
STATS_KEYS = ("factor_ms", "solve_ms", "iterations", "lambda_residual", "residual", "passes", "lambda_ms",
              "fronts_ms")


def plan_info(m, tet_part, n_parts: int) -> dict:
    """Symbolic analysis on the host only (no GPU): sizes of the FETI-DP plan."""
    pm, mh, maph = partitioned_dofmap(m, tet_part, n_parts, keep_handles=True)
    info = np.zeros(len(INFO_KEYS), np.int64)
    check(lib().emg_fetidp_plan_info(mh.h, maph.h, ptr(info), len(INFO_KEYS)), "emg_fetidp_plan_info")
    return dict(zip(INFO_KEYS, (int(v) for v in info)))


class FetiDP:
    """FETI-DP solver for the partitioned, gauged system of mesh ``m``.

    ``factor()`` runs the numeric phase for the mesh's materials and sources,
    ``solve()`` returns (x, SolverResult-like dict) with x in the partitioned
    map's numbering (``self.map.l2g``)."""

    def __init__(self, m, tet_part, n_parts: int, stream=None):
        self.m = m
        self.map, self._mesh, self._maph = partitioned_dofmap(m, tet_part, n_parts, keep_handles=True)
        self.h = C.c_void_p()
        check(lib().emg_fetidp_create(self._mesh.h, self._maph.h, stream, C.byref(self.h)), "emg_fetidp_create")

    def info(self) -> dict:
        v = np.zeros(len(INFO_KEYS), np.int64)
        check(lib().emg_fetidp_info(self.h, ptr(v), len(v)), "emg_fetidp_info")
        return dict(zip(INFO_KEYS, (int(a) for a in v)))

    def stats(self) -> dict:
        v = np.zeros(len(STATS_KEYS))
        check(lib().emg_fetidp_stats(self.h, ptr(v), len(v)), "emg_fetidp_stats")
        return dict(zip(STATS_KEYS, (float(a) for a in v)))

    def factor(self, flags: int = 0, nu=None, sigma=None) -> int:
        nu = np.ascontiguousarray(self.m.nu if nu is None else nu, np.float64)
        sg = np.ascontiguousarray(self.m.sigma if sigma is None else sigma, np.float64)
        arr, ns = _abi.sources_array(self.m.sources)
        return lib().emg_fetidp_factor(self.h, ptr(nu), ptr(sg), len(nu),
                                       C.cast(arr, C.c_void_p) if arr is not None else None, ns, flags)

    def solve(self, tol: float = 1e-10, max_iter: int = 500, precond: int = 2):
        """precond: 0 none, 1 Dirichlet with stiffness scaling, 2 Dirichlet with deluxe
        scaling, 3 the same with the S_DD blocks and face weights stored in FP32."""
        x = np.empty(self.map.n_dofs)
        cfg = _abi.KrylovConfig(tol, max_iter, precond)
        out = _abi.Result()
        rc = lib().emg_fetidp_solve(self.h, C.byref(cfg), ptr(x), 0, C.byref(out))
        return x, rc, out

    def solve_rhs(self, b, tol: float = 1e-10, max_iter: int = 500, precond: int = 2):
        """Solve with a caller's right-hand side (n_dofs, this map's numbering)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.empty(self.map.n_dofs)
        cfg = _abi.KrylovConfig(tol, max_iter, precond)
        out = _abi.Result()
        rc = lib().emg_fetidp_solve_rhs(self.h, C.byref(cfg), ptr(b), ptr(x), 0, C.byref(out))
        return x, rc, out

    def __del__(self, _abi=_abi):
        if getattr(self, "h", None) and _abi._LIB is not None:
            _abi._LIB.emg_fetidp_destroy(self.h)
            self.h = None


def gauged_map(m, gauge: int):
    """DOF map of the mesh under a tree gauge (emg_dof_build); returns the
    map handle owner, the mesh handle owner and the (T, 6 or 12) l2g."""
    mh = _MeshHandle(m)
    h = C.c_void_p()
    check(lib().emg_dof_build(mh.h, int(gauge), C.byref(h)), "emg_dof_build")
    ne, nf, nd = C.c_int64(), C.c_int64(), C.c_int64()
    lib().emg_dofmap_info(h, C.byref(ne), C.byref(nf), C.byref(nd))
    l2g = np.empty((m.n_tets, mesh.EDGES_OF_TYPE[m.elem_type]), np.int32)
    lib().emg_dofmap_export(h, ptr(l2g), None)
    return _MapHandle(h), mh, l2g, nd.value


def dual_layout(fd: "FetiDP") -> dict:
    """The multiplier layout of a FETI-DP solver (emg_fetidp_duals)."""
    info = fd.info()
    S, ne, nl = info["n_parts"], info["sum_nD"], info["n_lambda"]
    dual_off = np.empty(S + 1, np.int64)
    dual_lam = np.empty(max(ne, 1), np.int32)
    dual_sign = np.empty(max(ne, 1), np.int32)
    lam_entry = np.empty((max(nl, 1), 2), np.int32)
    check(lib().emg_fetidp_duals(fd.h, ptr(dual_off), ptr(dual_lam), ptr(dual_sign), ptr(lam_entry)),
          "emg_fetidp_duals")
    return {"n_parts": S, "n_entries": ne, "dual_off": dual_off, "dual_lam": dual_lam[:ne],
            "dual_sign": dual_sign[:ne], "lam_entry": lam_entry[:nl]}


class DirectSolver:
    """GPU sparse direct solver (nested dissection + multifrontal Cholesky,
    iterative refinement) for the gauged system of mesh ``m`` -- the
    SolverBackend role of the reference's MUMPS / Eigen LLT backends.  The DOF
    map comes from ``emg_dof_build(gauge)`` (the reference-exact ``ref`` gauge
    by default) or from a partitioned map when ``tet_part`` is given."""

    def __init__(self, m, gauge: int = _abi.GAUGE_REF, tet_part=None, n_parts: int = 0, stream=None):
        self.m = m
        if tet_part is not None:
            pm, self._mesh, self._maph = partitioned_dofmap(m, tet_part, n_parts, keep_handles=True)
            self.l2g, self.n_dofs = pm.l2g, pm.n_dofs
        else:
            self._maph, self._mesh, self.l2g, self.n_dofs = gauged_map(m, gauge)
        self.h = C.c_void_p()
        check(lib().emg_direct_create(self._mesh.h, self._maph.h, stream, C.byref(self.h)), "emg_direct_create")

    def info(self) -> dict:
        v = np.zeros(len(INFO_KEYS), np.int64)
        check(lib().emg_direct_info(self.h, ptr(v), len(v)), "emg_direct_info")
        return dict(zip(INFO_KEYS, (int(a) for a in v)))

    def factor(self, flags: int = 0, nu=None, sigma=None) -> int:
        nu = np.ascontiguousarray(self.m.nu if nu is None else nu, np.float64)
        sg = np.ascontiguousarray(self.m.sigma if sigma is None else sigma, np.float64)
        arr, ns = _abi.sources_array(self.m.sources)
        return lib().emg_direct_factor(self.h, ptr(nu), ptr(sg), len(nu),
                                       C.cast(arr, C.c_void_p) if arr is not None else None, ns, flags)

    def solve(self, b=None, tol: float = 1e-12, passes: int = 6):
        x = np.empty(self.n_dofs)
        bb = None if b is None else np.ascontiguousarray(b, np.float64)
        cfg = _abi.KrylovConfig(tol, passes, 0)
        out = _abi.Result()
        rc = lib().emg_direct_solve(self.h, C.byref(cfg), ptr(bb), ptr(x), 0, C.byref(out))
        return x, rc, out

    def __del__(self, _abi=_abi):
        if getattr(self, "h", None) and _abi._LIB is not None:
            _abi._LIB.emg_direct_destroy(self.h)
            self.h = None
