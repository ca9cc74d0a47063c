"""Host-side mirror of the reference's solve-path interfaces, backed by the
C ABI of libemagddm_b200 (CUDA kernels for sm_100a, host C++ numbering).

Names, argument meaning and error behaviour follow the reference classes:

=========================  ====================================================
this module                reference (Poofee/emagddm)
=========================  ====================================================
EMMeshData, BoundaryMarker include/fe_em/em_mesh_data.hpp:90-230
GlobalEdgeIDGenerator      src/fe_em/global_edge_id_generator.cpp:30-140
EMDOFManager               src/fe_em/em_dof_manager.cpp:29-626
MaterialProperties         include/numeric/em_element_integrator_base.hpp
EMAssembly                 src/numeric/em_assembly.cpp:144-420
CsrMatrix                  include/numeric/csr_matrix.hpp:31-259
CGConfig, CGSolver         src/numeric/iterative_solvers.cpp:64-503
BiCGSTABConfig, BiCGSTAB   src/numeric/iterative_solvers.cpp:820-1118
SolverStatus, SolverResult include/numeric/em_linear_solver.h:26-61
=========================  ====================================================

Errors: solver calls never raise; they return a SolverResult whose status
says what went wrong (as in the reference).  `assemble` returns False and
fills `getStats().error_message`.  Misuse of the numbering classes raises
ValueError / RuntimeError like the reference's std::invalid_argument /
std::runtime_error.
"""
from __future__ import annotations

import ctypes as C
import enum
import time
from dataclasses import dataclass, field

import numpy as np

from . import _abi, mesh
from ._abi import check, lib, ptr


class SolverStatus(enum.IntEnum):
    SUCCESS = 0
    NUMERICAL_ERROR = 1
    DIVERGED = 2
    MAX_ITER_REACHED = 3
    INVALID_INPUT = 4


class GaugeMode(enum.IntEnum):
    REF = _abi.GAUGE_REF
    BOUNDARY_FIRST = _abi.GAUGE_BOUNDARY_FIRST


@dataclass
class SolverResult:
    x: np.ndarray = None
    status: SolverStatus = SolverStatus.INVALID_INPUT
    iterations: int = 0
    residual_norm: float = 0.0
    solve_time_ms: float = 0.0
    error_msg: str = ""


@dataclass
class BoundaryMarker:
    """EMBoundaryMarker with vector (edge node pair) targets."""
    id: int
    bnd_type: str = "DIRICHLET"          # tool::BndType name
    dof_type: str = "VECTOR_EDGE_ONLY"
    target_ids: np.ndarray = None        # (k, 2) edge node pairs, or (k,) nodes
    value: float = 0.0
    name: str = ""


@dataclass
class EMMeshData:
    xyz: np.ndarray                      # (V, 3) node coordinates, node id = row
    tets: np.ndarray                     # (T, 4) TET4_EDGE or (T, 8) HEX8_EDGE elements
    material_id: np.ndarray = None       # (T,)
    boundary_markers: list = field(default_factory=list)
    # Element::dof_type per element (DOFType values or names); None = all
    # VECTOR_EDGE_ONLY
    dof_type: object = None

    @property
    def elem_type(self) -> int:
        """numeric::ElementType of the elements: TET4_EDGE (4 nodes) or HEX8_EDGE (8)."""
        return mesh.TYPE_OF_NODES[np.asarray(self.tets).shape[1]]

    def edges_per_element(self) -> int:
        return mesh.EDGES_OF_TYPE[self.elem_type]

    @classmethod
    def from_cube(cls, mesh) -> "EMMeshData":
        return cls(xyz=mesh.xyz, tets=mesh.tets, material_id=mesh.material,
                   boundary_markers=[BoundaryMarker(0, "DIRICHLET", "VECTOR_EDGE_ONLY",
                                                    mesh.dirichlet, 0.0, "outer_faces")])

    def getNodeCount(self) -> int:
        return int(self.xyz.shape[0])

    def getElementCount(self) -> int:
        return int(self.tets.shape[0])

    def dirichlet_pairs(self) -> np.ndarray:
        """Edge node pairs of every DIRICHLET marker on vector DOFs
        (EMDOFManager::markConstrainedDOFs, em_dof_manager.cpp:152-243)."""
        pairs = [np.asarray(m.target_ids, dtype=np.int32).reshape(-1, 2)
                 for m in self.boundary_markers
                 if m.bnd_type == "DIRICHLET" and m.dof_type in ("VECTOR_EDGE_ONLY", "MIXED_AV")
                 and m.target_ids is not None and np.asarray(m.target_ids).ndim == 2]
        return np.concatenate(pairs) if pairs else np.zeros((0, 2), np.int32)

    def dof_types(self):
        """Element::dof_type of every element as DOFType values, or None when
        every element is VECTOR_EDGE_ONLY."""
        if self.dof_type is None:
            return None
        names = {"SCALAR_ONLY": _abi.DOF_SCALAR_ONLY, "VECTOR_EDGE_ONLY": _abi.DOF_VECTOR_EDGE_ONLY,
                 "MIXED_AV": _abi.DOF_MIXED_AV}
        t = [names[v] if isinstance(v, str) else int(v) for v in np.asarray(self.dof_type).ravel()]
        t = np.ascontiguousarray(t, dtype=np.int32)
        if t.shape[0] != self.getElementCount():
            raise ValueError("dof_type needs one entry per element")
        return None if np.all(t == _abi.DOF_VECTOR_EDGE_ONLY) else t

    def scalar_dirichlet_nodes(self) -> np.ndarray:
        """Node IDs of every DIRICHLET marker on scalar DOFs
        (markConstrainedDOFs, em_dof_manager.cpp:163-177)."""
        nodes = [np.asarray(m.target_ids, dtype=np.int32).ravel() for m in self.boundary_markers
                 if m.bnd_type == "DIRICHLET" and m.dof_type in ("SCALAR_ONLY", "MIXED_AV")
                 and m.target_ids is not None and np.asarray(m.target_ids).ndim == 1]
        return np.concatenate(nodes) if nodes else np.zeros(0, np.int32)

    def hole_marker_count(self) -> int:
        """Markers the reference's heuristic counts as holes
        (MultiConnectedDomainDetector::analyzeBoundaryMarkers,
        multi_connected_domain.cpp:126-188)."""
        count = 0
        for m in self.boundary_markers:
            name = m.name.lower()
            if any(k in name for k in ("hole", "inner", "cavity", "孔")):
                count += 1
            if m.bnd_type in ("PERFECT_E", "PERFECT_H") and m.target_ids is not None:
                t = np.asarray(m.target_ids)
                limit = self.getNodeCount() // 2 if t.ndim == 1 else self.getElementCount() // 2
                if len(t) < limit and "hole" not in name:
                    count += 1
        return count


class _Mesh:
    """Owner of an emg_mesh handle."""

    def __init__(self, mesh: EMMeshData):
        L = lib()
        self.xyz = np.ascontiguousarray(mesh.xyz, dtype=np.float64)
        self.tets = np.ascontiguousarray(mesh.tets, dtype=np.int32)
        mat = mesh.material_id
        self.material = None if mat is None else np.ascontiguousarray(mat, dtype=np.int32)
        d = np.ascontiguousarray(mesh.dirichlet_pairs(), dtype=np.int32)
        self.h = C.c_void_p()
        check(L.emg_mesh_create_typed(mesh.elem_type, self.xyz.shape[0], ptr(self.xyz), self.tets.shape[0],
                                      ptr(self.tets), ptr(self.material), d.shape[0], ptr(d) if d.size else None,
                                      mesh.hole_marker_count(), C.byref(self.h)), "emg_mesh_create_typed")

    def __del__(self, _abi=_abi):
        if getattr(self, "h", None) and _abi._LIB is not None:
            _abi._LIB.emg_mesh_destroy(self.h)
            self.h = None


class GlobalEdgeIDGenerator:
    def __init__(self, mesh_data: EMMeshData):
        self.mesh_data = mesh_data
        self._mesh = None
        self._elem_edge = None
        self._edge_nodes = None
        self._lookup = None

    def generate(self) -> None:
        self._mesh = _Mesh(self.mesh_data)
        n = C.c_int64()
        check(lib().emg_edge_ids(self._mesh.h, None, None, C.byref(n)), "emg_edge_ids")
        T = self.mesh_data.getElementCount()
        self._elem_edge = np.empty((T, self.mesh_data.edges_per_element()), np.int32)
        self._edge_nodes = np.empty((n.value, 2), np.int32)
        check(lib().emg_edge_ids(self._mesh.h, ptr(self._elem_edge), ptr(self._edge_nodes), C.byref(n)),
              "emg_edge_ids")
        self._lookup = None

    def getNumGlobalEdges(self) -> int:
        return 0 if self._edge_nodes is None else int(self._edge_nodes.shape[0])

    def getElemLocalToGlobalEdge(self) -> np.ndarray:
        return self._elem_edge

    def getEdgeNodes(self) -> np.ndarray:
        return self._edge_nodes

    def getGlobalEdgeID(self, node1: int, node2: int) -> int:
        if self._lookup is None:
            self._lookup = {(int(a), int(b)): i for i, (a, b) in enumerate(self._edge_nodes)}
        return self._lookup.get((min(node1, node2), max(node1, node2)), -1)


class EMDOFManager:
    def __init__(self, mesh_data: EMMeshData, elem_local_to_global_edge=None,
                 edge_gen: GlobalEdgeIDGenerator | None = None):
        self.mesh_data = mesh_data
        self.edge_gen = edge_gen
        self._mesh = edge_gen._mesh if edge_gen is not None and edge_gen._mesh is not None else None
        self._l2g = None
        self._edge_dof = None
        self._n_free = 0
        self._n_dofs = 0
        self._gauged = False
        self._map = None

    def _run(self, gauge: int):
        if self._mesh is None:
            self._mesh = _Mesh(self.mesh_data)
        types = self.mesh_data.dof_types()
        if types is not None:
            return self._run_av(gauge, types)
        h = C.c_void_p()
        check(lib().emg_dof_build(self._mesh.h, gauge, C.byref(h)), "emg_dof_build")
        ne, nf, nd = C.c_int64(), C.c_int64(), C.c_int64()
        lib().emg_dofmap_info(h, C.byref(ne), C.byref(nf), C.byref(nd))
        l2g = np.empty((self.mesh_data.getElementCount(), self.mesh_data.edges_per_element()), np.int32)
        ed = np.empty(ne.value, np.int32)
        lib().emg_dofmap_export(h, ptr(l2g), ptr(ed))
        if self._map is not None:
            lib().emg_dofmap_destroy(self._map)
        self._map = h
        return l2g, ed, nf.value, nd.value

    def _run_av(self, gauge: int, types: np.ndarray):
        """Scalar / edge / A-V elements: rows of nodes + edges entries,
        Local2Global::indices padded with DOF_ABSENT."""
        md = self.mesh_data
        sd = np.ascontiguousarray(md.scalar_dirichlet_nodes(), dtype=np.int32)
        w = np.asarray(md.tets).shape[1] + md.edges_per_element()
        l2g = np.empty((md.getElementCount(), w), np.int32)
        ns, nf, nd = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().emg_dof_build_av(self._mesh.h, ptr(types), sd.size, ptr(sd) if sd.size else None, gauge,
                                     ptr(l2g), C.byref(ns), C.byref(nf), C.byref(nd)), "emg_dof_build_av")
        self._n_scalar_free = ns.value
        return l2g, None, nf.value, nd.value

    def build(self) -> None:
        self._l2g, self._edge_dof, self._n_free, self._n_dofs = self._run(_abi.GAUGE_NONE)
        self._gauged = False

    def applyTreeGauge(self, mode: GaugeMode = GaugeMode.REF) -> None:
        if self._l2g is None:
            raise RuntimeError("build() must be called before applyTreeGauge()")
        if self._gauged:
            return  # repeated calls are ignored (em_dof_manager.cpp:455-459)
        self._l2g, self._edge_dof, _, self._n_dofs = self._run(int(mode))
        self._gauged = True

    def getNumFreeDOFs(self) -> int:
        return self._n_dofs

    def getNumFreeDOFsBeforeGauge(self) -> int:
        return self._n_free

    def getElemLocalToGlobal(self) -> np.ndarray:
        """(T, epe) for edge-only meshes; with per-element DOF types (T,
        nodes + edges), each row Local2Global::indices padded with DOF_ABSENT."""
        return self._l2g

    def getElemLocalToGlobalList(self) -> list:
        """Local2Global::indices of every element, without padding."""
        return [row[row != _abi.DOF_ABSENT] for row in self._l2g]

    def getNumScalarFreeDOFs(self) -> int:
        """Free nodal (scalar) DOFs; they take equations 0 .. n - 1."""
        return getattr(self, "_n_scalar_free", 0)

    def getEdgeToDOF(self) -> np.ndarray:
        return self._edge_dof

    def mapReducedSolutionToFull(self, reduced) -> np.ndarray:
        if self._map is None:
            raise RuntimeError("mapReducedSolutionToFull needs an edge-only map built by build()")
        reduced = np.ascontiguousarray(reduced, dtype=np.float64)
        full = np.empty(self._edge_dof.shape[0])
        check(lib().emg_dofmap_expand(self._map, ptr(reduced), ptr(full)), "emg_dofmap_expand")
        return full

    def __del__(self, _abi=_abi):
        if getattr(self, "_map", None) is not None and _abi._LIB is not None:
            _abi._LIB.emg_dofmap_destroy(self._map)
            self._map = None


@dataclass
class MaterialProperties:
    mu: float = 4e-7 * np.pi
    sigma: float = 0.0
    epsilon: float = 8.854187817e-12


@dataclass
class AssemblyStats:
    assembly_time_ms: float = 0.0
    total_elements: int = 0
    free_dofs: int = 0
    nnz_stiffness: int = 0
    nnz_mass: int = 0
    is_symmetric_k: bool = True
    error_message: str = ""


class CsrMatrix:
    """Device CSR matrix (int32 row_ptr / col, fp64 values).  Host arrays are
    fetched lazily by get_row_ptr / get_col_indices / get_values."""

    def __init__(self, handle, owner=None, owned=False, host=None):
        self.h = handle
        self._owner = owner
        self._owned = owned
        self._host = host
        n, nnz = C.c_int64(), C.c_int64()
        check(lib().emg_csr_info(handle, C.byref(n), C.byref(nnz)), "emg_csr_info")
        self._n, self._nnz = n.value, nnz.value

    @classmethod
    def from_host(cls, n, row_ptr, col, val) -> "CsrMatrix":
        """CsrMatrix<double> built on the host (duplicates are summed)."""
        rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
        cc = np.ascontiguousarray(col, dtype=np.int32)
        vv = np.ascontiguousarray(val, dtype=np.float64)
        h = C.c_void_p()
        check(lib().emg_csr_create(n, ptr(rp), ptr(cc), ptr(vv), None, C.byref(h)), "emg_csr_create")
        return cls(h, owned=True)

    def rows(self) -> int:
        return self._n

    def cols(self) -> int:
        return self._n

    def nnz(self) -> int:
        return self._nnz

    def _fetch(self):
        if self._host is None:
            raise RuntimeError("host copy only available for assembled matrices")
        return self._host()

    def get_row_ptr(self):
        return self._fetch()[0]

    def get_col_indices(self):
        return self._fetch()[1]

    def get_values(self):
        return self._fetch()[2]

    def mat_vec(self, x):
        """y = A x on the GPU (device round trip through torch)."""
        import torch
        xd = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device="cuda")
        yd = torch.empty(self._n, dtype=torch.float64, device="cuda")
        check(lib().emg_spmv(self.h, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()),
                             C.c_void_p(torch.cuda.current_stream().cuda_stream)), "emg_spmv")
        return yd.cpu().numpy()

    def __del__(self, _abi=_abi):
        if getattr(self, "_owned", False) and _abi._LIB is not None and self.h:
            _abi._LIB.emg_csr_destroy(self.h)
            self.h = None


class EMAssembly:
    """GPU assembly of TET4_EDGE / HEX8_EDGE curl-curl systems (EMAssembly::assemble)."""

    def __init__(self):
        self._sys = None
        self._stats = AssemblyStats()
        self._host = None
        self.flags = 0

    def assemble(self, mesh_data: EMMeshData, elem_local_to_global, materials,
                 is_transient: bool = False, sources=(), flags: int = 0) -> bool:
        self.clear()
        L = lib()
        t0 = time.perf_counter()
        if mesh_data.getNodeCount() == 0 or mesh_data.getElementCount() == 0:
            self._stats.error_message = "mesh is empty"
            return False
        if not materials:
            self._stats.error_message = "materials list is empty"
            return False
        xyz = np.ascontiguousarray(mesh_data.xyz, dtype=np.float64)
        tets = np.ascontiguousarray(mesh_data.tets, dtype=np.int32)
        mat = None if mesh_data.material_id is None else np.ascontiguousarray(mesh_data.material_id, np.int32)
        l2g = np.ascontiguousarray(elem_local_to_global, dtype=np.int32)
        if l2g.shape[0] < tets.shape[0]:
            self._stats.error_message = "DOF map shorter than the element list"
            return False
        h = C.c_void_p()
        rc = L.emg_system_create_typed(mesh_data.elem_type, xyz.shape[0], ptr(xyz), tets.shape[0], ptr(tets),
                                       ptr(mat), ptr(l2g), 0, 0, None, C.byref(h))
        if rc != 0:
            self._stats.error_message = L.emg_last_error().decode()
            return False
        self._sys = h
        nu = np.array([1.0 / m.mu for m in materials])
        sigma = np.array([m.sigma for m in materials])
        arr, ns = _abi.sources_array(list(sources))
        fl = flags | (_abi.FLAG_MASS if is_transient else 0)
        rc = L.emg_system_assemble(h, ptr(nu), ptr(sigma), len(materials),
                                   C.cast(arr, C.c_void_p) if arr is not None else None, ns, fl, None)
        if rc != 0:
            self._stats.error_message = L.emg_last_error().decode()
            return False
        self.flags = fl
        n, nnz = C.c_int64(), C.c_int64()
        L.emg_system_info(h, C.byref(n), C.byref(nnz))
        self._stats = AssemblyStats(assembly_time_ms=(time.perf_counter() - t0) * 1e3,
                                    total_elements=tets.shape[0], free_dofs=n.value,
                                    nnz_stiffness=nnz.value,
                                    nnz_mass=nnz.value if is_transient else 0)
        return True

    def _export(self):
        if self._host is None:
            n, nnz = self._stats.free_dofs, self._stats.nnz_stiffness
            rp = np.empty(n + 1, np.int32)
            col = np.empty(nnz, np.int32)
            kv = np.empty(nnz)
            mv = np.empty(nnz) if self.flags & _abi.FLAG_MASS else None
            rhs = np.empty(n)
            check(lib().emg_system_export(self._sys, ptr(rp), ptr(col), ptr(kv), ptr(mv), ptr(rhs)),
                  "emg_system_export")
            self._host = (rp, col, kv, mv, rhs)
        return self._host

    def getStiffnessMatrix(self) -> CsrMatrix:
        return CsrMatrix(lib().emg_system_matrix(self._sys, 0), owner=self,
                         host=lambda: self._export()[:3])

    def getMassMatrix(self) -> CsrMatrix:
        h = lib().emg_system_matrix(self._sys, 1)
        if not h:
            raise RuntimeError("mass matrix was not assembled (is_transient=False)")
        return CsrMatrix(h, owner=self, host=lambda: (self._export()[0], self._export()[1], self._export()[3]))

    def getDampingMatrix(self) -> CsrMatrix:
        return self.getMassMatrix()  # C = M (magnetic_vector_3d_integrator.cpp:327-339)

    def getSourceVector(self) -> np.ndarray:
        return self._export()[4]

    def source_device_ptr(self) -> int:
        return lib().emg_system_rhs_device(self._sys)

    def getStats(self) -> AssemblyStats:
        return self._stats

    def clear(self):
        if self._sys is not None and _abi._LIB is not None:
            _abi._LIB.emg_system_destroy(self._sys)
        self._sys = None
        self._host = None

    def __del__(self, _abi=_abi):
        self.clear()


@dataclass
class IterativeSolverConfig:
    tolerance: float = 1e-8
    max_iterations: int = 1000
    residual_monitor_interval: int = 10
    preconditioner: str = "NONE"  # NONE | JACOBI | ILU0


CGConfig = IterativeSolverConfig
BiCGSTABConfig = IterativeSolverConfig


class _KrylovSolver:
    _bicg = False
    _base = ""

    def __init__(self, config: IterativeSolverConfig | None = None):
        self.config = config or IterativeSolverConfig()
        self._A = None
        self._history = []

    def set_config(self, config):
        self.config = config

    def get_config(self):
        return self.config

    def set_matrix(self, A: CsrMatrix):
        self._A = A
        self._history = []

    def get_solver_name(self) -> str:
        name = {"JACOBI": "Jacobi", "ILU0": "ILU0"}.get(str(self.config.preconditioner).upper(), "None")
        return f"{self._base}_{name}"

    def clear(self):
        self._A = None
        self._history = []

    def get_convergence_history(self):
        return list(self._history)

    def solve(self, b) -> SolverResult:
        res = SolverResult()
        if self._A is None:
            res.error_msg = "matrix not set; call set_matrix() first"
            return res
        b = np.ascontiguousarray(b, dtype=np.float64)
        if b.shape[0] != self._A.rows():
            res.error_msg = "right-hand side length does not match the matrix"
            return res
        # PreconditionerType values of iterative_solvers.h:59-76; unknown names
        # are rejected by the library rather than substituted
        kinds = {"NONE": _abi.PRECOND_NONE, "JACOBI": _abi.PRECOND_JACOBI, "ILU0": _abi.PRECOND_ILU0}
        cfg = _abi.KrylovConfig(self.config.tolerance, self.config.max_iterations,
                                kinds.get(str(self.config.preconditioner).upper(), -1))
        out = _abi.Result()
        x = np.empty_like(b)
        fn = lib().emg_bicgstab_solve if self._bicg else lib().emg_cg_solve
        rc = fn(self._A.h, ptr(b), ptr(x), C.byref(cfg), C.byref(out))
        res.x = x
        res.status = SolverStatus(out.status) if out.status <= 4 else SolverStatus.NUMERICAL_ERROR
        res.iterations = out.iterations
        res.residual_norm = out.residual_norm
        res.solve_time_ms = out.solve_time_ms
        if rc > 4 or rc == _abi.EMG_INVALID_INPUT:
            res.error_msg = lib().emg_last_error().decode()
        cap = max(out.iterations, 1)
        hist = np.empty(cap)
        k = lib().emg_last_history(self._A.h, ptr(hist), cap)
        every = max(1, self.config.residual_monitor_interval)
        self._history = [(i + 1, float(hist[i])) for i in range(k) if (i + 1) % every == 0 or i == 0]
        return res


class CGSolver(_KrylovSolver):
    _bicg = False
    _base = "CGSolver"


class BiCGSTABSolver(_KrylovSolver):
    _bicg = True
    _base = "BiCGSTABSolver"
