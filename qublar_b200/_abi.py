"""ctypes binding of the C ABI in include/qublar.h and include/qublar_synth.h.

The shared library is built in-tree (qublar_b200/libqublar_b200.so, by
``__graft_entry__.build()``). Loading fails loudly when it is missing: there is
no pure-Python or CPU fallback of the solver.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqublar_b200.so")

QB_OK = 0
STATUS_NAMES = {0: "QB_OK", 1: "QB_EINVAL", 2: "QB_ENOMEM", 3: "QB_EREFUSED", 4: "QB_ETIMEDOUT",
                5: "QB_ECUDA", 6: "QB_ENOTSUP", 7: "QB_ECANCELLED", 8: "QB_EBUSY"}
KIND_ISING = 1
KIND_RESIDUAL = 2
KIND_QUBO = 3
NOALLOC_SCRATCH_BYTES = 16 << 20
OPT_DEFER_UPLOAD = 1
OPT_RESID_CLUSTER = 2
OPT_TRACE = 4
REQ_PENDING, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = 0, 1, 2, 3, 4
RESID_LOCKSTEP = 1
RESID_CLUSTER = 2


class QBError(RuntimeError):
    """A non-OK qb_status, with the library's thread-local message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


# The C ABI takes plain pointers: it reads as many entries as the sizes and
# offsets in a descriptor say, and cannot see how long the caller's arrays
# are. The Python mirror knows, and refuses (QB_EINVAL) arrays shorter than
# their descriptor before any call.

def check_edge_lengths(kind: str, n: int, eu, ev, ew, h=None) -> None:
    if not (eu.size == ev.size == ew.size):
        raise QBError(1, f"{kind}: eu, ev and ew differ in length")
    if h is not None and h.size < n:
        raise QBError(1, f"{kind}: h is shorter than n")


def check_residual_lengths(d, w, row_ptr, ray, a, nbr_ptr, nbr, field=None) -> None:
    if row_ptr.size < 1:
        raise QBError(1, "residual: row_ptr is empty")
    n = row_ptr.size - 1
    if d.size != w.size:
        raise QBError(1, "residual: d and w differ in length")
    if nbr_ptr.size != n + 1:
        raise QBError(1, "residual: nbr_ptr and row_ptr differ in length")
    if not 0 <= int(row_ptr[-1]) <= min(ray.size, a.size):
        raise QBError(1, "residual: row_ptr[n] exceeds the length of ray or a")
    if not 0 <= int(nbr_ptr[-1]) <= nbr.size:
        raise QBError(1, "residual: nbr_ptr[n] exceeds the length of nbr")
    if field is not None and field.size < n:
        raise QBError(1, "residual: field is shorter than n")


class IsingDesc(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int64), ("eu", C.c_void_p), ("ev", C.c_void_p), ("ew", C.c_void_p)]


class QuboDesc(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int64), ("eu", C.c_void_p), ("ev", C.c_void_p), ("ew", C.c_void_p),
                ("h", C.c_void_p), ("offset", C.c_double)]


class ExportDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("voxel", C.c_double), ("lo", C.c_double * 3), ("n_vars", C.c_int32),
                ("var_voxel", C.c_void_p), ("p_void", C.c_void_p), ("p_void_noprior", C.c_void_p),
                ("truth", C.c_void_p), ("branches", C.c_void_p), ("n_branches", C.c_int32),
                ("lambda_", C.c_double), ("kappa", C.c_double)]


class ResidualDesc(C.Structure):
    _fields_ = [("n_vars", C.c_int32), ("n_rays", C.c_int32), ("d", C.c_void_p), ("w", C.c_void_p),
                ("row_ptr", C.c_void_p), ("ray", C.c_void_p), ("a", C.c_void_p), ("nbr_ptr", C.c_void_p),
                ("nbr", C.c_void_p), ("lambda_", C.c_double), ("kappa", C.c_double), ("field", C.c_void_p)]


class ScheduleC(C.Structure):
    _fields_ = [("t_hot", C.c_double), ("t_cold", C.c_double), ("anneal_sweeps", C.c_int32),
                ("hold_sweeps", C.c_int32), ("refresh_sweeps", C.c_int32)]


class Opts(C.Structure):
    _fields_ = [("stream", C.c_void_p), ("device", C.c_int32), ("flags", C.c_uint32)]


class ProblemInfo(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n", C.c_int32), ("nnz", C.c_int64), ("n_rays", C.c_int32),
                ("n_colours", C.c_int32), ("max_class", C.c_int32), ("field_bytes", C.c_int32),
                ("weight_bytes", C.c_int32), ("device_bytes", C.c_int64), ("sigma", C.c_double),
                ("w_min", C.c_double), ("field_bound", C.c_int64), ("variant", C.c_int32)]


class ResultInfo(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_branches", C.c_int32), ("sweeps", C.c_int32), ("launches", C.c_int32),
                ("anneal_ms", C.c_float), ("total_ms", C.c_float), ("attempts", C.c_int64),
                ("max_drift", C.c_double), ("accepted", C.c_int64), ("max_energy_error", C.c_double)]


class TomoParams(C.Structure):
    _fields_ = [("target_bits", C.c_int32), ("target_rays", C.c_int32), ("voxel", C.c_double),
                ("half_base", C.c_double), ("height", C.c_double), ("n_detectors", C.c_int32),
                ("det", C.c_double * 12), ("n_theta", C.c_int32), ("n_phi", C.c_int32),
                ("theta_min", C.c_double), ("theta_max", C.c_double), ("phi_half", C.c_double),
                ("sub_rays", C.c_int32), ("room_radius", C.c_double), ("mu_rock", C.c_double), ("void_center", C.c_double * 3),
                ("void_side", C.c_double), ("exposure", C.c_double), ("min_open", C.c_double),
                ("lambda_", C.c_double), ("kappa", C.c_double), ("seed", C.c_uint64)]


class BatchItem(C.Structure):
    _fields_ = [("problem", C.c_void_p), ("schedule", ScheduleC), ("n_branches", C.c_uint32),
                ("seed_offset", C.c_uint64)]


class BatchConfig(C.Structure):
    _fields_ = [("threads", C.c_int32), ("smem_bytes", C.c_int32), ("max_group", C.c_int32), ("ctas", C.c_int32)]


class BatchInfo(C.Structure):
    _fields_ = [("items", C.c_int32), ("work_items", C.c_int32), ("global_items", C.c_int32),
                ("threads", C.c_int32), ("smem_bytes", C.c_int32), ("max_group", C.c_int32), ("ctas", C.c_int32),
                ("launches", C.c_int32), ("attempts", C.c_int64), ("anneal_ms", C.c_float), ("total_ms", C.c_float)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_int64), ("max_active", C.c_int32),
                ("residual_streams", C.c_int32), ("tick_target_us", C.c_int32), ("use_graph", C.c_int32),
                ("batch", BatchConfig), ("max_pending", C.c_int32), ("coop_parts", C.c_int32)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("kind", C.c_int32), ("n", C.c_int32),
                ("n_branches", C.c_int32), ("sweeps", C.c_int32), ("attempts", C.c_int64),
                ("device_bytes", C.c_int64), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "completed", "failed", "cancelled", "pending", "active", "ticks",
                                          "bytes_in_use", "peak_bytes", "budget_bytes", "attempts_done")]


class EnumResult(C.Structure):
    _fields_ = [("log_z", C.c_double), ("e_min", C.c_double), ("x_min", C.c_uint64), ("mean_energy", C.c_double),
                ("states", C.c_uint64)]


_P = C.c_void_p
# name -> (restype, argtypes)
SIGNATURES = {
    "qb_status_string": (C.c_char_p, [C.c_int]),
    "qb_last_error": (C.c_char_p, []),
    "qb_abi_version": (C.c_int32, []),
    "qb_device_count": (C.c_int32, []),
    "qb_problem_create_ising": (C.c_int, [C.POINTER(IsingDesc), C.POINTER(Opts), C.POINTER(_P)]),
    "qb_problem_create_residual": (C.c_int, [C.POINTER(ResidualDesc), C.POINTER(Opts), C.POINTER(_P)]),
    "qb_problem_create_qubo": (C.c_int, [C.POINTER(QuboDesc), C.POINTER(Opts), C.POINTER(_P)]),
    "qb_problem_destroy": (None, [_P]),
    "qb_problem_info_get": (C.c_int, [_P, C.POINTER(ProblemInfo)]),
    "qb_problem_colouring": (C.c_int, [_P, _P, _P, C.POINTER(C.c_int32)]),
    "qb_schedule_scaled": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(ScheduleC)]),
    "qb_solve": (C.c_int, [_P, C.POINTER(ScheduleC), C.c_uint32, C.c_uint64, C.POINTER(Opts), C.POINTER(_P)]),
    "qb_result_info_get": (C.c_int, [_P, C.POINTER(ResultInfo)]),
    "qb_result_branches": (C.c_int, [_P, _P]),
    "qb_result_energies_i64": (C.c_int, [_P, _P]),
    "qb_result_fields_i64": (C.c_int, [_P, _P]),
    "qb_result_energies_f64": (C.c_int, [_P, _P]),
    "qb_result_marginals": (C.c_int, [_P, _P]),
    "qb_result_tristate": (C.c_int, [_P, C.c_float, C.c_float, _P]),
    "qb_result_energy_trace": (C.c_int, [_P, _P]),
    "qb_result_destroy": (None, [_P]),
    "qb_energies_ising": (C.c_int, [_P, _P, C.c_int32, _P]),
    "qb_energies_residual": (C.c_int, [_P, _P, C.c_int32, _P]),
    "qb_energies_qubo": (C.c_int, [_P, _P, C.c_int32, _P]),
    "qb_solve_residual_noalloc": (C.c_int, [_P, C.POINTER(ScheduleC), C.c_uint32, C.c_uint64, _P, _P, _P]),
    "qb_metropolis_check": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, _P, _P, _P]),
    "qb_device_trim": (C.c_int, [C.c_int32]),
    "qb_batch_autotune": (C.c_int, [C.POINTER(BatchItem), C.c_int32, C.c_int32, C.POINTER(Opts),
                                    C.POINTER(BatchConfig)]),
    "qb_solve_batch": (C.c_int, [C.POINTER(BatchItem), C.c_int32, C.POINTER(BatchConfig), C.POINTER(Opts),
                                 C.POINTER(_P)]),
    "qb_batch_info_get": (C.c_int, [_P, C.POINTER(BatchInfo)]),
    "qb_batch_branches": (C.c_int, [_P, C.c_int32, _P]),
    "qb_batch_energies_i64": (C.c_int, [_P, C.c_int32, _P]),
    "qb_batch_fields_i64": (C.c_int, [_P, C.c_int32, _P]),
    "qb_batch_marginals": (C.c_int, [_P, C.c_int32, _P]),
    "qb_batch_destroy": (None, [_P]),
    "qb_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(_P)]),
    "qb_server_submit": (C.c_int, [_P, _P, C.POINTER(ScheduleC), C.c_uint32, C.c_uint64, C.POINTER(C.c_uint64)]),
    "qb_server_poll": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_int32)]),
    "qb_server_wait": (C.c_int, [_P, C.c_uint64, C.c_int32]),
    "qb_server_cancel": (C.c_int, [_P, C.c_uint64]),
    "qb_server_request_info": (C.c_int, [_P, C.c_uint64, C.POINTER(RequestInfo)]),
    "qb_server_result_branches": (C.c_int, [_P, C.c_uint64, _P]),
    "qb_server_result_marginals": (C.c_int, [_P, C.c_uint64, _P]),
    "qb_server_result_energies_i64": (C.c_int, [_P, C.c_uint64, _P]),
    "qb_server_result_energies_f64": (C.c_int, [_P, C.c_uint64, _P]),
    "qb_server_release": (C.c_int, [_P, C.c_uint64]),
    "qb_server_stats_get": (C.c_int, [_P, C.POINTER(ServerStats)]),
    "qb_server_destroy": (None, [_P]),
    "qb_parse_rudy": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(_P)]),
    "qb_graph_desc": (C.c_int, [_P, C.POINTER(IsingDesc)]),
    "qb_graph_destroy": (None, [_P]),
    "qb_freeze_rock": (C.c_int, [C.POINTER(ResidualDesc), C.c_double, C.POINTER(Opts), C.POINTER(_P)]),
    "qb_freeze_info": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "qb_freeze_kept": (C.c_int, [_P, _P]),
    "qb_freeze_reduced": (C.c_int, [_P, C.POINTER(ResidualDesc)]),
    "qb_freeze_destroy": (None, [_P]),
    "qb_roi_qubo": (C.c_int, [C.POINTER(ResidualDesc), _P, C.c_int32, _P, _P, _P]),
    "qb_enumerate_qubo": (C.c_int, [C.c_int32, _P, _P, C.c_double, C.POINTER(Opts), C.POINTER(EnumResult), _P]),
    "qb_colour_ising": (C.c_int, [C.POINTER(IsingDesc), _P, _P, C.POINTER(C.c_int32)]),
    "qb_colour_residual": (C.c_int, [C.POINTER(ResidualDesc), _P, _P, C.POINTER(C.c_int32)]),
    "qb_tomo_params_default": (None, [C.POINTER(TomoParams)]),
    "qb_synth_tomography": (C.c_int, [C.POINTER(TomoParams), C.POINTER(_P)]),
    "qb_synth_tomography_device": (C.c_int, [C.POINTER(TomoParams), C.POINTER(Opts), C.POINTER(_P)]),
    "qb_tomo_sizes": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                C.POINTER(C.c_int64)]),
    "qb_tomo_arrays": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "qb_tomo_desc": (C.c_int, [_P, C.POINTER(ResidualDesc)]),
    "qb_tomo_cells": (C.c_int, [_P, _P, _P]),
    "qb_tomo_destroy": (None, [_P]),
    "qb_write_ising_out": (C.c_int, [C.c_char_p, C.POINTER(ExportDesc)]),
    "qb_write_roi_text": (C.c_int, [C.c_char_p, C.c_int32, _P, _P, _P, _P, _P]),
    "qb_parse_qubo_text": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(_P)]),
    "qb_qubo_text_info": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "qb_qubo_text_arrays": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "qb_qubo_text_desc": (C.c_int, [_P, C.POINTER(QuboDesc)]),
    "qb_qubo_text_destroy": (None, [_P]),
    "qb_write_qubo_text": (C.c_int, [C.c_char_p, C.c_int32, C.c_int64, C.c_double, C.c_double, C.c_double, _P, _P,
                                     _P, _P, _P]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded library (loaded once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() (make -C qublar_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != QB_OK:
        raise QBError(status, lib().qb_last_error().decode("utf-8", "replace"))


def ptr(a) -> int | None:
    """Address of a contiguous numpy array (None for None)."""
    if a is None:
        return None
    return a.ctypes.data
