"""ctypes binding of the C ABI in include/beta_gpu.h.

Loads the in-tree libbeta_gpu.so.  There is no fallback: if the library is
missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libbeta_gpu.so")

# status codes
OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_STATE = 3
MAXIT = 4
BREAKDOWN = 5
ERR_NEGDIAG = 6
ERR_ZERODIAG = 7
ERR_OOM = 8
REJECTED = 9
TIMEOUT = 10
ERR_NOT_FINITE = 11
ERR_LOAD_ON_RESTRAINED = 12
ERR_UNSUPPORTED = 13
ERR_TOO_LARGE = 14
NOALLOC_MAX_ROWS = 262144

# system exchange formats
FMT_ADDRESS_LOWER = 1
FMT_ADDRESS_UPPER = 2
FMT_COMPRESSED_ROW = 3
FMT_CSR_ASCII = 4
FMT_CSR_BINARY = 5

# server request states
REQ_QUEUED = 0
REQ_RUNNING = 1
REQ_DONE = 2
REQ_REJECTED = 3
REQ_CANCELLED = 4
REQ_FAILED = 5

QUAD4_PSTRESS = 1
HEX8_ELASTIC = 2
HEX8_HEAT = 3
QUAD4_HEAT = 4

ASM_K = 1
ASM_MBAR = 2
ASM_TANGENT = 3

FP64 = 0
FP32 = 1

MODE_FP64 = 0
MODE_MPIR = 1
PRECOND_JACOBI = 0
PRECOND_BLOCK_JACOBI = 1
STOP_REF = 0
STOP_RB = 1

STATUS_NAMES = {
    0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_STATE", 4: "MAXIT", 5: "BREAKDOWN",
    6: "ERR_NEGDIAG", 7: "ERR_ZERODIAG", 8: "ERR_OOM", 9: "REJECTED", 10: "TIMEOUT",
    11: "ERR_NOT_FINITE", 12: "ERR_LOAD_ON_RESTRAINED", 13: "ERR_UNSUPPORTED", 14: "ERR_TOO_LARGE",
}


class SolveOpts(C.Structure):
    _fields_ = [
        ("mode", C.c_int), ("precond", C.c_int), ("stop_rule", C.c_int), ("maxit", C.c_int),
        ("tol", C.c_double), ("inner_tol", C.c_double), ("max_outer", C.c_int),
        ("use_last_solution", C.c_int), ("check_every", C.c_int), ("reserved", C.c_int),
    ]


class SolveStats(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("iterations", C.c_int), ("outer_iterations", C.c_int), ("reserved", C.c_int),
        ("final_norm", C.c_double), ("true_rel_residual", C.c_double), ("ms_solve", C.c_double),
        ("ms_spmv_avg", C.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class NewtonOpts(C.Structure):
    _fields_ = [("max_residual", C.c_double), ("max_newton", C.c_int), ("use_last_solution", C.c_int),
                ("solve", SolveOpts)]


class NewtonStats(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("linear_iterations", C.c_int),
                ("reserved", C.c_int), ("max_residual", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class System(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("ndim", C.c_int), ("nnode", C.c_int), ("nelem", C.c_int), ("nnpe", C.c_int),
        ("ndof_per_node", C.c_int), ("integration_order", C.c_int), ("ngroups", C.c_int), ("nparams", C.c_int),
        ("reserved", C.c_int),
        ("xyz", C.c_void_p), ("conn", C.c_void_p), ("first_dof", C.c_void_p), ("group_params", C.c_void_p),
        ("elem_group", C.c_void_p), ("restrained", C.c_void_p), ("prescribed", C.c_void_p), ("load", C.c_void_p),
    ]


# Every exported symbol with its signature (kept in step with include/beta_gpu.h).
_P = C.c_void_p
_I = C.c_int
_D = C.c_double
SIGNATURES = {
    "beta_gpu_create": (_I, [C.POINTER(_P), _I]),
    "beta_gpu_destroy": (_I, [_P]),
    "beta_gpu_last_error": (C.c_char_p, [_P]),
    "beta_gpu_version": (_I, []),
    "beta_gpu_set_stream": (_I, [_P, _P]),
    "beta_gpu_set_zero_diagonal": (_I, [_P, _D]),
    "beta_gpu_counters": (_I, [_P, C.POINTER(C.c_longlong), _I]),
    "beta_gpu_mesh_upload": (_I, [_P, _I, _I, _I, _P, _I, _I, _P, _P, _I, _I]),
    "beta_gpu_materials_upload": (_I, [_P, _I, _I, _P, _P]),
    "beta_gpu_bc_upload": (_I, [_P, _P, _P, _P]),
    "beta_gpu_build_pattern": (_I, [_P, C.POINTER(C.c_longlong)]),
    "beta_gpu_set_block_runs": (_I, [_P, _I]),
    "beta_gpu_block_layout": (_I, [_P, C.POINTER(C.c_longlong), _I]),
    "beta_gpu_set_operator_cache": (_I, [_P, _I]),
    "beta_gpu_pattern_lower": (_I, [_P, _P, _P]),
    "beta_gpu_pattern_lower_host": (_I, [_I, _I, _I, _I, _P, _P, _P, C.POINTER(C.c_longlong), _P, _P]),
    "beta_gpu_assemble": (_I, [_P, _I, _I, _D, _D]),
    "beta_gpu_matrix_lower_values": (_I, [_P, _I, _P, _P]),
    "beta_gpu_solve": (_I, [_P, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "beta_gpu_solve_rhs": (_I, [_P, _P, _P, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "beta_gpu_read_mesh": (_I, [C.c_char_p, _I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), C.POINTER(_I), _P,
                                _P]),
    "beta_gpu_write_mesh": (_I, [C.c_char_p, _I, _I, _I, _P, _I, _I, _P, _I]),
    "beta_gpu_surface_flux_load": (_I, [_I, _I, _P, _I, _P, _P, _P, _I, _P]),
    "beta_gpu_parse_element_groups": (_I, [C.c_char_p, _I, _P, _P]),
    "beta_gpu_write_lower": (_I, [C.c_char_p, _I, _I, _P, _P, _P]),
    "beta_gpu_read_lower": (_I, [C.c_char_p, _I, C.POINTER(_I), C.POINTER(C.c_longlong), _P, _P, _P]),
    "beta_gpu_export_matrix": (_I, [_P, _I, _I, C.c_char_p]),
    "beta_gpu_element_outputs": (_I, [_P, _P, _P, _P]),
    "beta_gpu_download": (_I, [_P, _P]),
    "beta_gpu_matvec": (_I, [_P, _I, _P, _P]),
    "beta_gpu_internal_force": (_I, [_P, _P, _P]),
    "beta_gpu_internal_force_nonlinear": (_I, [_P, _P, _P]),
    "beta_gpu_set_solution": (_I, [_P, _P]),
    "beta_gpu_newton": (_I, [_P, C.POINTER(NewtonOpts), C.POINTER(NewtonStats), _P]),
    "beta_gpu_heat_set_state": (_I, [_P, _P]),
    "beta_gpu_heat_run": (_I, [_P, _D, _D, _I, C.POINTER(SolveOpts), C.POINTER(SolveStats), C.POINTER(_I)]),
    "beta_gpu_heat_get_state": (_I, [_P, _P]),
    "beta_gpu_csr_pcg_device": (_I, [_I, _P, _P, _P, _P, _P, _I, _D, _I, _P, C.POINTER(SolveStats)]),
    "beta_gpu_batch_create": (_I, [C.POINTER(_P), _I, C.c_longlong, _I]),
    "beta_gpu_batch_destroy": (_I, [_P]),
    "beta_gpu_batch_last_error": (C.c_char_p, [_P]),
    "beta_gpu_batch_add": (_I, [_P, _I, _I, _I, _P, _I, _I, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P, C.POINTER(_I)]),
    "beta_gpu_batch_add_many": (_I, [_P, _I, C.POINTER(System), _I, C.POINTER(_I)]),
    "beta_gpu_batch_run": (_I, [_P, C.POINTER(SolveOpts), _I, C.POINTER(_I)]),
    "beta_gpu_batch_result": (_I, [_P, _I, _P, C.POINTER(SolveStats)]),
    "beta_gpu_batch_remove": (_I, [_P, _I]),
    "beta_gpu_batch_tune": (_I, [_P, _I, _I]),
    "beta_gpu_batch_autotune": (_I, [_P, C.POINTER(SolveOpts), _I, C.POINTER(_I), C.POINTER(_I)]),
    "beta_gpu_batch_reset": (_I, [_P]),
    "beta_gpu_batch_set_switch": (_I, [_P, _I]),
    "beta_gpu_batch_set_slice": (_I, [_P, C.c_longlong]),
    "beta_gpu_batch_test_barrier": (_I, [_P, C.c_longlong, _I]),
    "beta_gpu_gang_plan": (_I, [_I, C.POINTER(C.c_longlong), C.POINTER(_I), _I, _I, _I, C.POINTER(_I)]),
    "beta_gpu_batch_info": (_I, [_P, C.POINTER(C.c_longlong), _I]),
    "beta_gpu_server_create": (_I, [C.POINTER(_P), _I, C.c_longlong, _I, C.POINTER(SolveOpts), _I, _I, _I]),
    "beta_gpu_server_destroy": (_I, [_P]),
    "beta_gpu_server_last_error": (C.c_char_p, [_P]),
    "beta_gpu_server_submit": (_I, [_P, _I, _I, _I, _P, _I, _I, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P,
                                    C.POINTER(C.c_longlong)]),
    "beta_gpu_server_poll": (_I, [_P, C.c_longlong, _I, C.POINTER(_I), C.POINTER(_I), _P, C.POINTER(SolveStats),
                                  C.POINTER(_D), _I]),
    "beta_gpu_server_cancel": (_I, [_P, C.c_longlong]),
    "beta_gpu_server_set_slice": (_I, [_P, C.c_longlong]),
    "beta_gpu_server_stats": (_I, [_P, C.POINTER(C.c_longlong), _I]),
    "beta_gpu_csr_pcg_device_noalloc": (_I, [_I, _P, _P, _P, _P, _P, _I, _D, _I, _P, C.POINTER(SolveStats)]),
}

_lib = None


def load(path: str | None = None):
    """Loads (once) and returns the library; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"CUDA extension not built: {p} is missing (run python -m betanoox_b200.build)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class BetaGpuError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status
