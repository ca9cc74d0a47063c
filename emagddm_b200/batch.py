"""Batched many-instance curl-curl solves.

Many independent cube problems are assembled as ONE system: the union of the
(disjoint) meshes, material ids and DOF numbers offset per instance, and a
per-tet source map so each instance keeps its own current box.  The matrix is
then block diagonal with one block per instance, and
``emg_batch_cg_solve_device`` runs Jacobi-PCG on every block in lockstep
inside a single CUDA graph (per-block scalars, statuses and iteration counts).

The instance set of the "batched many-instance" workload: instance i draws
its grid size n ~ U{8..32} from seed 7 + i and gets a random axis-aligned
box with mu_r in [1, 1000] plus a uniform J_z in a random sub-box
(:func:`emagddm_b200.mesh.random_instance`).
"""
from __future__ import annotations

import ctypes as C
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import _abi, api, mesh


def instance_sizes(count: int, seed0: int = 7, nmin: int = 8, nmax: int = 32):
    return [int(np.random.default_rng(seed0 + i).integers(nmin, nmax + 1)) for i in range(count)]


def make_instances(count: int, seed0: int = 7, nmin: int = 8, nmax: int = 32):
    sizes = instance_sizes(count, seed0, nmin, nmax)
    return [mesh.random_instance(n, seed0 + i) for i, n in enumerate(sizes)]


def number_instance(m, gauge=api.GaugeMode.REF) -> np.ndarray:
    md = api.EMMeshData.from_cube(m)
    dm = api.EMDOFManager(md)
    dm.build()
    dm.applyTreeGauge(gauge)
    return np.ascontiguousarray(dm.getElemLocalToGlobal(), np.int32)


@dataclass
class Batch:
    xyz: np.ndarray
    tets: np.ndarray
    material: np.ndarray
    l2g: np.ndarray
    nu: np.ndarray
    sigma: np.ndarray
    sources: list
    tet_source: np.ndarray
    block_row_ptr: np.ndarray   # int64, n_instances + 1
    instances: list
    l2g_each: list

    @property
    def n_rows(self) -> int:
        return int(self.block_row_ptr[-1])


def build_batch(instances, threads: int = 8) -> Batch:
    """Union of the instances' meshes with per-instance offsets."""
    with ThreadPoolExecutor(threads) as ex:  # the C++ numbering releases the GIL
        l2g_each = list(ex.map(number_instance, instances))
    xyz, tets, mat, l2g, nu, sigma, src, tsrc = [], [], [], [], [], [], [], []
    rows = [0]
    node_off = 0
    for i, (m, l) in enumerate(zip(instances, l2g_each)):
        n_dofs = int(l.max()) + 1 if l.size and l.max() >= 0 else 0
        xyz.append(m.xyz)
        tets.append(m.tets + node_off)
        mat.append(m.material + len(nu))
        nu.extend(m.nu)
        sigma.extend(m.sigma)
        ll = l.copy()
        ll[ll >= 0] += rows[-1]
        l2g.append(ll)
        src.extend(m.sources)
        tsrc.append(np.full(m.n_tets, len(src) - len(m.sources) if m.sources else -1, np.int32))
        rows.append(rows[-1] + n_dofs)
        node_off += m.n_nodes
    return Batch(xyz=np.ascontiguousarray(np.concatenate(xyz)),
                 tets=np.ascontiguousarray(np.concatenate(tets), np.int32),
                 material=np.ascontiguousarray(np.concatenate(mat), np.int32),
                 l2g=np.ascontiguousarray(np.concatenate(l2g), np.int32),
                 nu=np.asarray(nu, np.float64), sigma=np.asarray(sigma, np.float64), sources=src,
                 tet_source=np.ascontiguousarray(np.concatenate(tsrc), np.int32),
                 block_row_ptr=np.asarray(rows, np.int64), instances=list(instances), l2g_each=l2g_each)


class BatchSystem:
    """Assembled block-diagonal system of a Batch on the GPU."""

    def __init__(self, b: Batch, stream=None, resident: dict | None = None):
        L = _abi.lib()
        self.batch = b
        self.h = C.c_void_p()
        if resident is None:
            rc = L.emg_system_create(b.xyz.shape[0], _abi.ptr(b.xyz), b.tets.shape[0], _abi.ptr(b.tets),
                                     _abi.ptr(b.material), _abi.ptr(b.l2g), b.n_rows, stream,
                                     C.byref(self.h))
        else:
            rc = L.emg_system_create_device(b.xyz.shape[0], resident["xyz"], b.tets.shape[0],
                                            resident["tets"], resident["material"], resident["l2g"],
                                            b.n_rows, stream, C.byref(self.h))
        _abi.check(rc, "emg_system_create")
        _abi.check(L.emg_system_set_source_map(self.h, _abi.ptr(b.tet_source)), "emg_system_set_source_map")
        arr, ns = _abi.sources_array(b.sources)
        _abi.check(L.emg_system_assemble(self.h, _abi.ptr(b.nu), _abi.ptr(b.sigma), len(b.nu),
                                         C.cast(arr, C.c_void_p) if arr is not None else None, ns, 0,
                                         stream), "emg_system_assemble")

    def solve(self, x_d, tol=1e-8, max_iter=20000, precond=_abi.PRECOND_JACOBI, stream=None):
        """Lockstep batched Jacobi-PCG; x_d: device pointer (int) of n_rows doubles."""
        L = _abi.lib()
        b = self.batch
        nb = len(b.instances)
        res = (_abi.Result * nb)()
        cfg = _abi.KrylovConfig(tol, max_iter, precond)
        rc = L.emg_batch_cg_solve_device(L.emg_system_matrix(self.h, 0), nb, _abi.ptr(b.block_row_ptr),
                                         C.c_void_p(L.emg_system_rhs_device(self.h)), C.c_void_p(x_d),
                                         C.byref(cfg), stream, res)
        return rc, [dict(status=r.status, iterations=r.iterations, residual=r.residual_norm,
                         ms=r.solve_time_ms) for r in res]

    def export(self):
        L = _abi.lib()
        n, nnz = C.c_int64(), C.c_int64()
        L.emg_system_info(self.h, C.byref(n), C.byref(nnz))
        rp = np.empty(n.value + 1, np.int32)
        col = np.empty(nnz.value, np.int32)
        kv = np.empty(nnz.value)
        rhs = np.empty(n.value)
        _abi.check(L.emg_system_export(self.h, _abi.ptr(rp), _abi.ptr(col), _abi.ptr(kv), None, _abi.ptr(rhs)),
                   "emg_system_export")
        return rp, col, kv, rhs

    def __del__(self, _abi=_abi):
        if getattr(self, "h", None) and _abi._LIB is not None:
            _abi._LIB.emg_system_destroy(self.h)
            self.h = None
