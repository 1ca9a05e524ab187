"""ctypes binding of libgraphene_b200.so (include/graphene_gpu.h).

The library is built in-tree by ``graphene_b200.build``; importing this
module never compiles anything and raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgraphene_b200.so"

GR_OK = 0
GR_EINVAL = 1
GR_ENOMEM = 2
GR_EPARSE = 3
GR_ENOTCONV = 4
GR_EBREAKDOWN = 5
GR_ETIMEOUT = 6
GR_ECUDA = 7
GR_EUNSUPPORTED = 8
GR_EIO = 9
GR_ENONFINITE = 10
GR_ECANCELED = 11

FLOAT32, FLOAT64, TWOFLOAT32 = 0, 1, 2
NORM_L1, NORM_L2, NORM_LINF, NORM_NONE = 0, 1, 2, 3
PART_AUTO, PART_CONTIGUOUS, PART_RCB, PART_BFS, PART_EXPLICIT, PART_MULTILEVEL = 0, 1, 2, 3, 4, 5


class Stats(C.Structure):
    _fields_ = [
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
        ("b_norm", C.c_double),
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("singular", C.c_int32),
        ("status", C.c_int32),
        ("inner_iterations", C.c_int32),
        ("reserved", C.c_int32),
        ("solve_ms", C.c_double),
    ]


class MatrixInfo(C.Structure):
    _fields_ = [
        ("num_rows", C.c_int64),
        ("num_off_diag", C.c_int64),
        ("num_tiles", C.c_int64),
        ("num_halo_total", C.c_int64),
        ("max_tile_rows", C.c_int64),
        ("num_lower_levels_total", C.c_int64),
        ("num_upper_levels_total", C.c_int64),
        ("value_type", C.c_int32),
        ("format", C.c_int32),
        ("multicolor_recommended", C.c_int32),
        ("reserved", C.c_int32),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("slots", C.c_int32), ("device", C.c_int32), ("hbm_budget_bytes", C.c_int64)]


class RequestTimes(C.Structure):
    _fields_ = [
        ("arrival_ms", C.c_double),
        ("admitted_ms", C.c_double),
        ("finished_ms", C.c_double),
        ("footprint_bytes", C.c_int64),
        ("cache_hit", C.c_int32),
        ("slot", C.c_int32),
        ("solve_start_ms", C.c_double),
    ]


vp = C.c_void_p
i64 = C.c_int64
i32 = C.c_int32
P = C.POINTER

# name -> (restype, argtypes)
SIGNATURES = {
    "gr_last_error": (C.c_char_p, []),
    "gr_version": (C.c_int, []),
    "gr_launch_count": (i64, []),
    "gr_host_matrix_from_coo": (C.c_int, [i64, i64, vp, vp, vp, i64, C.c_int, vp, vp, C.c_int, P(vp)]),
    "gr_host_matrix_poisson": (C.c_int, [i64, i64, i64, i64, C.c_int, C.c_int, P(vp)]),
    "gr_host_matrix_from_ldu": (C.c_int, [i64, i64, vp, vp, vp, vp, vp, i64, C.c_int, vp, vp, C.c_int, P(vp)]),
    "gr_host_matrix_ldu_mesh": (C.c_int, [i64, i64, i64, C.c_uint64, C.c_uint64, C.c_uint64, i64, C.c_int,
                                          C.c_int, P(vp)]),
    "gr_host_matrix_get_ldu": (C.c_int, [vp, P(i64), vp, vp, vp, vp, vp]),
    "gr_host_matrix_load_mm": (C.c_int, [C.c_char_p, i64, C.c_int, C.c_int, P(vp)]),
    "gr_host_matrix_generate": (C.c_int, [C.c_int, i64, i64, i64, vp, C.c_uint64, i64, C.c_int,
                                          C.c_int, P(vp)]),
    "gr_random_vector": (C.c_int, [C.c_uint64, i64, C.c_int, C.c_double, C.c_double, vp]),
    "gr_host_matrix_global_crs": (C.c_int, [vp, vp, vp, vp, vp]),
    "gr_host_matrix_destroy": (None, [vp]),
    "gr_host_matrix_astype": (C.c_int, [vp, C.c_int, P(vp)]),
    "gr_host_matrix_get_info": (C.c_int, [vp, P(MatrixInfo)]),
    "gr_host_matrix_row_to_tile": (C.c_int, [vp, vp]),
    "gr_host_matrix_edge_cut": (C.c_int, [vp, P(i64)]),
    "gr_host_matrix_tile_sizes": (C.c_int, [vp, vp]),
    "gr_host_matrix_local_to_global": (C.c_int, [vp, vp]),
    "gr_host_matrix_local_crs": (C.c_int, [vp, vp, vp, vp, vp]),
    "gr_host_matrix_levels": (C.c_int, [vp, vp, vp]),
    "gr_host_matrix_check_ilu_stream": (C.c_int, [vp, C.c_int, C.c_int, P(i32), P(i64)]),
    "gr_host_matrix_load_vector_mm": (C.c_int, [vp, C.c_char_p, C.c_int, vp]),
    "gr_host_matrix_check_ilu_ring": (C.c_int, [vp, C.c_int, C.c_int, i64, i32, i32, P(i64), P(i64), P(i32)]),
    "gr_host_matrix_check_gs_ring": (C.c_int, [vp, C.c_int, C.c_int, i64, i32, P(i64), P(i64), P(i32), P(i32)]),
    "gr_host_matrix_set_spmv_layout": (C.c_int, [vp, i32]),
    "gr_host_matrix_check_spmv_layout": (C.c_int, [vp, i32, P(i32), P(i64), P(i64), P(i64)]),
    "gr_matrix_spmv_layout": (C.c_int, [vp, P(i32), P(i64), P(i64)]),
    "gr_host_matrix_decompose_vector": (C.c_int, [vp, vp, vp, C.c_int]),
    "gr_host_matrix_compose_vector": (C.c_int, [vp, vp, vp, C.c_int]),
    "gr_matrix_create": (C.c_int, [vp, P(vp)]),
    "gr_matrix_destroy": (None, [vp]),
    "gr_matrix_set_stream": (C.c_int, [vp, vp]),
    "gr_matrix_get_info": (C.c_int, [vp, P(MatrixInfo)]),
    "gr_spmv": (C.c_int, [vp, vp, vp, C.c_int]),
    "gr_residual": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, vp, C.c_int, C.c_int]),
    "gr_vector_norm": (C.c_int, [vp, C.c_int, vp, C.c_int, P(C.c_double)]),
    "gr_vector_norms_noalloc": (C.c_int, [vp, i64, i64, i64, C.c_int, C.c_int, vp, vp]),
    "gr_solver_time_repeated": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, i32, P(C.c_float)]),
    "gr_matrix_tune_spmv": (C.c_int, [vp, C.c_int, i32, P(i32), P(i32), P(i32), P(C.c_float)]),
    "gr_matrix_time_spmv": (C.c_int, [vp, vp, vp, C.c_int, i32, i32, P(C.c_float)]),
    "gr_server_create": (C.c_int, [P(ServerConfig), P(vp)]),
    "gr_server_submit": (C.c_int, [vp, vp, C.c_char_p, vp, C.c_int, P(C.c_uint64)]),
    "gr_server_wait": (C.c_int, [vp, C.c_uint64, C.c_double, vp, P(Stats), P(RequestTimes)]),
    "gr_server_counters": (C.c_int, [vp, P(i64), P(i64), P(i64), P(i64), P(i64)]),
    "gr_server_destroy": (None, [vp]),
    "gr_server_cancel": (C.c_int, [vp, C.c_uint64, P(i32)]),
    "gr_matrix_inject_status": (C.c_int, [vp, i32]),
    "gr_host_matrix_generate_like": (C.c_int, [vp, C.c_int, i64, i64, i64, P(C.c_double), C.c_uint64, P(vp)]),
    "gr_host_matrix_structure_key": (C.c_int, [vp, P(C.c_uint64)]),
    "gr_matrix_update_values": (C.c_int, [vp, vp]),
    "gr_solver_refresh": (C.c_int, [vp]),
    "gr_matrix_update_global_values": (C.c_int, [vp, vp, vp]),
    "gr_host_matrix_generate_values": (C.c_int, [vp, C.c_int, i64, i64, i64, P(C.c_double), C.c_uint64, vp, vp]),
    "gr_server_submit_values": (C.c_int, [vp, vp, vp, vp, C.c_char_p, vp, C.c_int, P(C.c_uint64)]),
    "gr_batch_create": (C.c_int, [P(vp), i32, C.c_char_p, P(vp)]),
    "gr_batch_solve_host": (C.c_int, [vp, P(vp), P(vp), C.c_int, P(Stats)]),
    "gr_batch_destroy": (None, [vp]),
    "gr_selftest_wait_timeout": (C.c_int, [P(i32), P(i64)]),
    "gr_decompose_vector": (C.c_int, [vp, vp, vp, C.c_int]),
    "gr_compose_vector": (C.c_int, [vp, vp, vp, C.c_int]),
    "gr_solver_create": (C.c_int, [vp, C.c_char_p, P(vp)]),
    "gr_solver_destroy": (None, [vp]),
    "gr_solve": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, P(Stats)]),
    "gr_solve_host": (C.c_int, [vp, vp, C.c_int, vp, C.c_int, P(Stats)]),
    "gr_solver_phi": (C.c_int, [vp, vp, C.c_int]),
    "gr_solver_name": (C.c_int, [vp, C.c_char_p, C.c_size_t]),
    "gr_config_parse": (C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]),
}

_lib = None


class GrapheneError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m graphene_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != GR_OK:
        raise GrapheneError(rc, lib().gr_last_error().decode(errors="replace"))
