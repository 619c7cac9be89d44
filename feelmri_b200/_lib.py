"""ctypes binding of libfeelmri_b200.so (the C ABI in include/feelmri_b200.h).

The shared library is built in-tree by feelmri_b200.build.  Importing this
module does not need a GPU; creating a context does.  There is no fallback:
when the library is missing or the device is not a B200, calls raise.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfeelmri_b200.so"

FM_OK = 0
FM_ERR_SHAPE = 1
FM_ERR_DTYPE = 2
FM_ERR_CUDA = 3
FM_ERR_NOMEM = 4
FM_ERR_TIMEOUT = 5
FM_ERR_ARG = 6
FM_ERR_UNSUPPORTED = 7
FM_ERR_CANCELLED = 8

FM_NUM_NONE = 0
FM_NUM_PYFLOAT = 1
FM_NUM_F32 = 2
FM_NUM_F64 = 3

FM_MOTION_NONE = 0
FM_MOTION_TERMS = 1
FM_MOTION_TABLE = 2

FM_TERM_POD = 0
FM_TERM_POD_VELOCITY = 1
FM_TERM_RESPIRATORY = 2
FM_MAX_MOTION_TERMS = 4

FM_PREC_F32 = 0
FM_PREC_F64 = 1
FM_PREC_BF16X3 = 2

_p = C.c_void_p
_i64 = C.c_int64
_i32 = C.c_int32


class MotionTerm(C.Structure):
    _fields_ = [
        ("kind", _i32),
        ("n_modes", _i32),
        ("modes", _p),
        ("pp_c", _p),
        ("pp_x", _p),
        ("pp_k", _i32),
        ("pp_intervals", _i32),
        ("timeshift", C.c_double),
        ("timeshift_kind", _i32),
        ("period_kind", _i32),
        ("period", C.c_double),
        ("direction", C.c_float * 3),
        ("extrapolate", _i32),
    ]


class Motion(C.Structure):
    _fields_ = [
        ("kind", _i32),
        ("n_terms", _i32),
        ("terms", MotionTerm * FM_MAX_MOTION_TERMS),
        ("table", _p),
        ("table_calls", _i64),
    ]


class BlochArgs(C.Structure):
    _fields_ = [
        ("n_pos", _i64),
        ("n_time", _i64),
        ("r0", _p),
        ("T1", _p),
        ("T2", _p),
        ("delta_B", _p),
        ("M0", C.c_float),
        ("gamma", C.c_float),
        ("rf", _p),
        ("G", _p),
        ("dt", _p),
        ("Mxy0", _p),
        ("Mz0", _p),
        ("motion", C.POINTER(Motion)),
        ("Mxy_hist", _p),
        ("Mz_hist", _p),
        ("Mxy_final", _p),
        ("Mz_final", _p),
        ("Mxy_carry", _p),
        ("final_stride", _i64),
    ]


class BlochBlock(C.Structure):
    _fields_ = [
        ("offset", _i64),
        ("n_time", _i64),
        ("empty", C.c_int32),
        ("store", C.c_int32),
        ("timeshift", C.c_double * FM_MAX_MOTION_TERMS),
        ("timeshift_kind", C.c_int32 * FM_MAX_MOTION_TERMS),
    ]


class BlochSequenceArgs(C.Structure):
    _fields_ = [
        ("n_pos", _i64),
        ("r0", _p),
        ("T1", _p),
        ("T2", _p),
        ("delta_B", _p),
        ("M0", C.c_float),
        ("gamma", C.c_float),
        ("n_blocks", C.c_int32),
        ("blocks", C.POINTER(BlochBlock)),
        ("n_samples", _i64),
        ("rf", _p),
        ("G", _p),
        ("dt", _p),
        ("Mxy0", _p),
        ("Mz0", _p),
        ("motion", C.POINTER(Motion)),
        ("n_store", C.c_int32),
        ("Mxy_out", _p),
        ("Mz_out", _p),
        ("Mxy_carry", _p),
        ("Mz_carry", _p),
    ]


class SignalArgs(C.Structure):
    _fields_ = [
        ("n_nodes", _i64),
        ("n_vencs", _i64),
        ("n_ro", _i64),
        ("n_lines", _i64),
        ("n_kz", _i64),
        ("m_rows", _i64),
        ("m_cols", _i64),
        ("m_nnz", _i64),
        ("m_indptr", _p),
        ("m_indices", _p),
        ("m_data", _p),
        ("kx", _p),
        ("ky", _p),
        ("kz", _p),
        ("t", _p),
        ("r0", _p),
        ("phi", _p),
        ("T2", _p),
        ("Mxy", _p),
        ("motion", C.POINTER(Motion)),
        ("out", _p),
    ]


class MassArgs(C.Structure):
    _fields_ = [
        ("n_elems", _i64),
        ("nodes_per_elem", _i32),
        ("elems", _p),
        ("n_nodes", _i64),
        ("nodes", _p),
        ("n_qpoints", _i32),
        ("qweights", _p),
        ("tabulated", _p),
    ]


# name -> (restype, argtypes)
class TcTuning(C.Structure):
    """fm_tc_tuning: work-unit shape of the batched tensor-core Signal."""
    _fields_ = [("split_nodes", C.c_int32), ("kz_cap", C.c_int32), ("reserved", C.c_int32 * 2)]


SIGNATURES = {
    "fm_ctx_create": (C.c_int, [C.c_int, C.POINTER(_p)]),
    "fm_ctx_destroy": (C.c_int, [_p]),
    "fm_ctx_set_stream": (C.c_int, [_p, _p]),
    "fm_ctx_synchronize": (C.c_int, [_p]),
    "fm_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "fm_abi_version": (C.c_int, []),
    "fm_launch_count": (C.c_int64, []),
    "fm_ctx_timing_enable": (C.c_int, [_p, C.c_int]),
    "fm_ctx_timing_reset": (C.c_int, [_p]),
    "fm_ctx_timing_query": (C.c_int, [_p, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "fm_pod_tensordot_f32": (C.c_int, [_p, _p, _p, _i64, _i64, _i64, _p]),
    "fm_pod_tensordot_f64": (C.c_int, [_p, _p, _p, _i64, _i64, _i64, _p]),
    "fm_pod_build_workspace_size": (C.c_int, [_i64, C.c_int32, C.c_int32, C.POINTER(C.c_size_t)]),
    "fm_pod_gram_f32": (C.c_int, [_p, _p, _i64, C.c_int32, _p, _p, C.c_size_t]),
    "fm_pod_gram_f64": (C.c_int, [_p, _p, _i64, C.c_int32, _p, _p, C.c_size_t]),
    "fm_pod_project_f32": (C.c_int, [_p, _p, _i64, C.c_int32, _p, C.c_int32, _p, _p, _p, C.c_size_t]),
    "fm_pod_project_f64": (C.c_int, [_p, _p, _i64, C.c_int32, _p, C.c_int32, _p, _p, _p, C.c_size_t]),
    "fm_coil_expand": (C.c_int, [_p, _p, _p, _i64, _i64, _p]),
    "fm_motion_eval": (C.c_int, [_p, C.POINTER(Motion), _i64, _p, _i64, _p, _p, C.c_size_t]),
    "fm_motion_eval_workspace_size": (C.c_int, [C.POINTER(Motion), _i64, _i64, C.POINTER(C.c_size_t)]),
    "fm_bloch_solve_f32": (C.c_int, [_p, C.POINTER(BlochArgs), _p, C.c_size_t]),
    "fm_bloch_workspace_size": (C.c_int, [C.POINTER(BlochArgs), C.POINTER(C.c_size_t)]),
    "fm_bloch_solve_f32_noalloc": (C.c_int, [_p, C.POINTER(BlochArgs)]),
    "fm_bloch_sequence_f32": (C.c_int, [_p, C.POINTER(BlochSequenceArgs), _p, C.c_size_t]),
    "fm_bloch_sequence_workspace_size": (C.c_int, [C.POINTER(BlochSequenceArgs), C.POINTER(C.c_size_t)]),
    "fm_signal": (C.c_int, [_p, C.POINTER(SignalArgs), C.c_int, _p, C.c_size_t]),
    "fm_signal_enqueue": (C.c_int, [_p, C.POINTER(SignalArgs), C.c_int, _p, C.c_size_t]),
    "fm_signal_status": (C.c_int, [_p, C.POINTER(SignalArgs), C.c_int, _p, C.c_size_t]),
    "fm_signal_workspace_size": (C.c_int, [C.POINTER(SignalArgs), C.c_int, C.POINTER(C.c_size_t)]),
    "fm_signal_count_time_runs": (C.c_int64, [_p, _i64, C.c_int]),
    "fm_signal_batch_workspace_size": (C.c_int, [C.POINTER(SignalArgs), C.c_int, C.POINTER(C.c_size_t)]),
    "fm_signal_batch_enqueue": (C.c_int, [_p, C.POINTER(SignalArgs), C.c_int, C.POINTER(TcTuning), _p, C.c_size_t]),
    "fm_signal_batch_status": (C.c_int, [_p, C.POINTER(SignalArgs), C.c_int, _p, C.c_size_t]),
    "fm_selftest_wait": (C.c_int, [_p, C.c_uint64]),
    "fm_mass_assemble": (C.c_int, [_p, C.POINTER(MassArgs), C.c_int, C.POINTER(_i64), _p, _p, _p, _i64, _p,
                                   C.c_size_t]),
    "fm_mass_lumped": (C.c_int, [_p, C.POINTER(MassArgs), C.c_int, _p, _p, C.c_size_t]),
    "fm_mass_workspace_size": (C.c_int, [C.POINTER(MassArgs), C.c_int, C.POINTER(C.c_size_t)]),
}


class FeelMRIError(RuntimeError):
    """Raised when an entry point of libfeelmri_b200 returns a failure status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[fm status {code}] {message}")
        self.code = code


_lib = None
_lib_lock = threading.Lock()


def lib() -> C.CDLL:
    """Loads the shared library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise ImportError(
                    f"{LIB_PATH.name} is not built; run `python -m feelmri_b200.build` (nvcc, sm_100a)")
            handle = C.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(2048)
    lib().fm_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != FM_OK:
        msg = last_error()
        if status in (FM_ERR_SHAPE,):
            raise ValueError(f"[fm status {status}] {msg}")
        raise FeelMRIError(status, msg)


_ctx_lock = threading.Lock()
_ctxs: dict[tuple[int, int], int] = {}


def bind_stream(device: int, stream_handle: int) -> int:
    """The library context (an opaque pointer) for work on `stream_handle` of
    `device`.  One context per (device, stream), so host threads that drive
    different streams never share one."""
    key = (device, int(stream_handle or 0))
    with _ctx_lock:
        h = _ctxs.get(key)
        if h is None:
            out = _p()
            check(lib().fm_ctx_create(device, C.byref(out)))
            h = out.value
            check(lib().fm_ctx_set_stream(h, _p(stream_handle)))
            _ctxs[key] = h
        return h


def launch_count() -> int:
    return int(lib().fm_launch_count())


def timing(ctx: int, on: bool) -> None:
    check(lib().fm_ctx_timing_enable(ctx, 1 if on else 0))


def timing_reset(ctx: int) -> None:
    check(lib().fm_ctx_timing_reset(ctx))


def timing_query(ctx: int, prefix: str) -> tuple[float, int]:
    ms = C.c_double()
    n = C.c_int64()
    check(lib().fm_ctx_timing_query(ctx, prefix.encode(), C.byref(ms), C.byref(n)))
    return ms.value, n.value
