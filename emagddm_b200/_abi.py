"""ctypes binding of libemagddm_b200.so (the C ABI in include/emagddm_b200.h).

The library is built in-tree (emagddm_b200/build.py) and loaded from the
package directory.  There is no fallback: if the library is missing the
import fails with an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libemagddm_b200.so")

EMG_SUCCESS, EMG_NUMERICAL_ERROR, EMG_DIVERGED, EMG_MAX_ITER_REACHED, EMG_INVALID_INPUT = 0, 1, 2, 3, 4
EMG_ERR_CUDA, EMG_ERR_TIMEOUT, EMG_ERR_NOMEM, EMG_ERR_INTERNAL = 5, 6, 7, 8
GAUGE_NONE, GAUGE_REF, GAUGE_BOUNDARY_FIRST = -1, 0, 1
FLAG_MASS, FLAG_NO_EDGE_SIGNS, FLAG_PIOLA_LITERAL, FLAG_QUAD3_LITERAL = 1, 2, 4, 8
ELEM_TET4_EDGE, ELEM_HEX8_EDGE, ELEM_PRISM6_EDGE, ELEM_PYRAMID5_EDGE = 0, 1, 2, 3
DOF_SCALAR_ONLY, DOF_VECTOR_EDGE_ONLY, DOF_MIXED_AV, DOF_ABSENT = 0, 1, 2, -2
PRECOND_NONE, PRECOND_JACOBI, PRECOND_ILU0 = 0, 1, 2

I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
VP = C.c_void_p
H = C.c_void_p  # opaque handle


class Source(C.Structure):
    _fields_ = [("kind", C.c_int32), ("j", C.c_double * 3), ("p", C.c_double * 6)]


class KrylovConfig(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_int32),
                ("preconditioner", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32),
                ("residual_norm", C.c_double), ("solve_time_ms", C.c_double)]


# Exported symbols and their ctypes signatures (argtypes, restype).
SIGNATURES = {
    "emg_abi_version": ([], C.c_int32),
    "emg_last_error": ([], C.c_char_p),
    "emg_mesh_create": ([C.c_int64, VP, C.c_int64, VP, VP, C.c_int64, VP, C.c_int32,
                         C.POINTER(H)], C.c_int),
    "emg_mesh_create_typed": ([C.c_int32, C.c_int64, VP, C.c_int64, VP, VP, C.c_int64, VP, C.c_int32,
                               C.POINTER(H)], C.c_int),
    "emg_mesh_elem_type": ([H, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
    "emg_mesh_destroy": ([H], None),
    "emg_mesh_read_gmsh": ([C.c_char_p, VP, C.c_int32, C.POINTER(H)], C.c_int),
    "emg_mesh_info": ([H, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                       C.POINTER(C.c_int32)], C.c_int),
    "emg_mesh_export": ([H, VP, VP, VP, VP], C.c_int),
    "emg_mesh_material_tags": ([H, VP], C.c_int),
    "emg_edge_ids": ([H, VP, VP, C.POINTER(C.c_int64)], C.c_int),
    "emg_dof_build": ([H, C.c_int32, C.POINTER(H)], C.c_int),
    "emg_dof_build_device": ([C.c_int32, C.c_int64, C.c_int64, VP, C.c_int64, VP, C.c_int32, C.c_int32, VP,
                              C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64), VP], C.c_int),
    "emg_dof_build_av": ([H, VP, C.c_int64, VP, C.c_int32, VP, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                          C.POINTER(C.c_int64)], C.c_int),
    "emg_dofmap_info": ([H, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "emg_dofmap_export": ([H, VP, VP], C.c_int),
    "emg_dofmap_expand": ([H, VP, VP], C.c_int),
    "emg_dofmap_destroy": ([H], None),
    "emg_dof_build_partitioned": ([H, VP, C.c_int32, C.POINTER(H)], C.c_int),
    "emg_dofmap_partition_info": ([H, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int64), VP],
                                  C.c_int),
    "emg_system_create": ([C.c_int64, VP, C.c_int64, VP, VP, VP, C.c_int64, VP, C.POINTER(H)], C.c_int),
    "emg_system_create_device": ([C.c_int64, VP, C.c_int64, VP, VP, VP, C.c_int64, VP,
                                  C.POINTER(H)], C.c_int),
    "emg_system_create_typed": ([C.c_int32, C.c_int64, VP, C.c_int64, VP, VP, VP, C.c_int64, C.c_int32, VP,
                                 C.POINTER(H)], C.c_int),
    "emg_system_assemble": ([H, VP, VP, C.c_int32, VP, C.c_int32, C.c_int32, VP], C.c_int),
    "emg_system_set_source_map": ([H, VP], C.c_int),
    "emg_system_info": ([H, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "emg_system_export": ([H, VP, VP, VP, VP, VP], C.c_int),
    "emg_system_matrix": ([H, C.c_int32], H),
    "emg_system_rhs_device": ([H], VP),
    "emg_system_destroy": ([H], None),
    "emg_csr_create": ([C.c_int64, VP, VP, VP, VP, C.POINTER(H)], C.c_int),
    "emg_csr_create_device": ([C.c_int64, C.c_int64, VP, VP, VP, VP, C.POINTER(H)], C.c_int),
    "emg_csr_info": ([H, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "emg_csr_destroy": ([H], None),
    "emg_spmv": ([H, VP, VP, VP], C.c_int),
    "emg_cg_solve": ([H, VP, VP, C.POINTER(KrylovConfig), C.POINTER(Result)], C.c_int),
    "emg_cg_solve_device": ([H, VP, VP, C.POINTER(KrylovConfig), VP, C.POINTER(Result)], C.c_int),
    "emg_bicgstab_solve": ([H, VP, VP, C.POINTER(KrylovConfig), C.POINTER(Result)], C.c_int),
    "emg_bicgstab_solve_device": ([H, VP, VP, C.POINTER(KrylovConfig), VP, C.POINTER(Result)], C.c_int),
    "emg_system_solve": ([H, C.c_int32, C.POINTER(KrylovConfig), VP, C.c_int32, VP,
                          C.POINTER(Result)], C.c_int),
    "emg_cg_kernel_times": ([H, C.c_int32, VP, VP], C.c_int),
    "emg_test_set_barrier_spins": ([C.c_int32], C.c_int),
    "emg_tune_enable": ([C.c_int32], C.c_int),
    "emg_aedt_read": ([C.c_char_p, C.POINTER(H)], C.c_int),
    "emg_aedt_info": ([H, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
    "emg_aedt_material": ([H, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                           C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
    "emg_aedt_bh_curve": ([H, C.c_int32, VP, VP, C.c_int32], C.c_int),
    "emg_aedt_object": ([H, C.c_int32, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(C.c_int32)],
                        C.c_int),
    "emg_aedt_boundary": ([H, C.c_int32, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32, C.c_char_p, C.c_int32],
                          C.c_int),
    "emg_aedt_destroy": ([H], None),
    "emg_tune_report": ([C.c_char_p, C.c_int32], C.c_int32),
    "emg_test_tc_tile": ([C.c_int32, C.c_int32, C.c_int32, VP, C.c_int64, VP, C.c_int64, VP, C.c_int64, VP],
                         C.c_int),
    "emg_system_combine": ([H, C.c_double, C.c_double, C.POINTER(H)], C.c_int),
    "emg_batch_cg_solve_device": ([H, C.c_int32, VP, VP, VP, C.POINTER(KrylovConfig), VP, VP], C.c_int),
    "emg_cg_solve_noalloc": ([C.c_int64, C.c_int64, VP, VP, VP, VP, VP, C.POINTER(KrylovConfig), VP,
                              C.POINTER(Result)], C.c_int),
    "emg_csr_solver_format": ([H, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "emg_last_history": ([H, VP, C.c_int32], C.c_int),
    "emg_fetidp_plan_info": ([H, H, VP, C.c_int32], C.c_int),
    "emg_fetidp_create": ([H, H, VP, C.POINTER(H)], C.c_int),
    "emg_fetidp_factor": ([H, VP, VP, C.c_int32, VP, C.c_int32, C.c_int32], C.c_int),
    "emg_fetidp_solve": ([H, C.POINTER(KrylovConfig), VP, C.c_int32, C.POINTER(Result)], C.c_int),
    "emg_fetidp_solve_rhs": ([H, C.POINTER(KrylovConfig), VP, VP, C.c_int32, C.POINTER(Result)], C.c_int),
    "emg_fetidp_info": ([H, VP, C.c_int32], C.c_int),
    "emg_fetidp_stats": ([H, VP, C.c_int32], C.c_int),
    "emg_fetidp_destroy": ([H], None),
    "emg_fetidp_learned_init": ([H, C.c_uint64], C.c_int),
    "emg_fetidp_learned_train": ([H, C.c_int32, VP, VP, C.c_float, C.POINTER(C.c_double)], C.c_int),
    "emg_fetidp_learned_params": ([H, VP, C.POINTER(C.c_int64), C.c_int32], C.c_int),
    "emg_fetidp_apply": ([H, C.c_int32, VP, VP], C.c_int),
    "emg_fetidp_lambda_rhs": ([H, VP, VP], C.c_int),
    "emg_fetidp_duals": ([H, VP, VP, VP, VP], C.c_int),
    "emg_direct_create": ([H, H, VP, C.POINTER(H)], C.c_int),
    "emg_direct_factor": ([H, VP, VP, C.c_int32, VP, C.c_int32, C.c_int32], C.c_int),
    "emg_direct_solve": ([H, C.POINTER(KrylovConfig), VP, VP, C.c_int32, C.POINTER(Result)], C.c_int),
    "emg_direct_info": ([H, VP, C.c_int32], C.c_int),
    "emg_direct_destroy": ([H], None),
}

_LIB = None


class EmgError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().emg_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "or `make -C emagddm_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _LIB = L
    return _LIB


def check(code: int, where: str) -> int:
    if code != EMG_SUCCESS:
        raise EmgError(code, where)
    return code


def ptr(a):
    """Host numpy array -> void* (None passes NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.c_void_p)


def sources_array(sources):
    if not sources:
        return None, 0
    arr = (Source * len(sources))()
    for k, s in enumerate(sources):
        arr[k].kind = int(s.kind)
        for i in range(3):
            arr[k].j[i] = float(s.j[i])
        for i in range(6):
            arr[k].p[i] = float(s.p[i])
    return arr, len(sources)


def tune_report() -> dict:
    """The autotuner's decisions so far (emg_tune_report), as a dict."""
    import json
    n = lib().emg_tune_report(None, 0)
    buf = C.create_string_buffer(int(n))
    lib().emg_tune_report(buf, n)
    return json.loads(buf.value.decode() or "{}")
