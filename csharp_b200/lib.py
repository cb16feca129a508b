"""ctypes binding of ``libswgb200.so`` (the C ABI declared in ``include/swgb200.h``).

The product path has no CPU fallback: loading fails loudly when the library is missing, and
every call that reports a non-zero status raises :class:`SwError` with the context's message.
"""
import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libswgb200.so"

SW_OK, SW_E_ARG, SW_E_OOM, SW_E_CUDA, SW_E_TIMEOUT, SW_E_UNSUPPORTED, SW_E_STATE, SW_E_IO, SW_E_THROWS = range(9)
SW_PROTEIN, SW_NUCLEIC = 0, 1
SW_DIST_PERCENT_IDENTITY, SW_DIST_KIMURA2, SW_DIST_JUKES_CANTOR, SW_DIST_MIN_MAX_NORM_SCORE = 0, 1, 2, 3
SW_MODE_SWG_MPI, SW_MODE_SWG_MS, SW_MODE_NW = 0, 1, 2
SW_LANES_AUTO, SW_LANES_16, SW_LANES_32 = 0, 16, 32

STATUS_NAMES = {SW_OK: "SW_OK", SW_E_ARG: "SW_E_ARG", SW_E_OOM: "SW_E_OOM", SW_E_CUDA: "SW_E_CUDA",
                SW_E_TIMEOUT: "SW_E_TIMEOUT", SW_E_UNSUPPORTED: "SW_E_UNSUPPORTED",
                SW_E_STATE: "SW_E_STATE", SW_E_IO: "SW_E_IO", SW_E_THROWS: "SW_E_THROWS"}

# Every symbol include/swgb200.h declares (checked against the built library by the tests).
EXPORTS = [
    "sw_create", "sw_destroy", "sw_last_error", "sw_version", "sw_upload_sequences",
    "sw_compute_block", "sw_compute_block_device", "sw_align_pair", "sw_all_pairs_device",
    "sw_all_pairs", "sw_last_rerun_count", "sw_synchronize", "sw_parse_scoring_matrix",
    "sw_builtin_scoring_matrix", "sw_parse_fasta", "sw_partition_ranges", "sw_block_is_computed",
    "sw_write_full_matrix", "sw_write_ms_block", "sw_read_ms_block_dims", "sw_read_ms_block_values",
    "sw_measure_int_peak", "sw_set_option", "sw_compute_rank_blocks", "sw_compute_rows", "sw_query",
    "sw_compute_block_static", "sw_submit_job", "sw_poll", "sw_serve_stats", "sw_serve_drain",
    "sw_autotune", "sw_align_strings",
]


class SwError(RuntimeError):
    def __init__(self, status, message=""):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class sw_config(C.Structure):
    _fields_ = [("mode", C.c_int32), ("alignment_type", C.c_int32), ("distance_fn", C.c_int32),
                ("gap_open", C.c_float), ("gap_extension", C.c_float),
                ("scores", C.c_int16 * (128 * 128)), ("device", C.c_int32), ("lanes", C.c_int32)]


class sw_pair_result(C.Structure):
    _fields_ = [("score", C.c_float), ("end1", C.c_int32), ("end2", C.c_int32),
                ("start1", C.c_int32), ("start2", C.c_int32), ("identity", C.c_int32),
                ("similarity", C.c_int32), ("gaps", C.c_int32), ("length", C.c_int32),
                ("distance", C.c_int16), ("reserved", C.c_int16)]


class sw_job_info(C.Structure):
    _fields_ = [("status", C.c_int32), ("queries", C.c_int32), ("pairs", C.c_int64), ("cells", C.c_int64),
                ("submit_s", C.c_double), ("admit_s", C.c_double), ("done_s", C.c_double),
                ("waves", C.c_int32), ("reserved", C.c_int32)]


class sw_serve_counters(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("waves", C.c_int64), ("cells", C.c_int64),
                ("active", C.c_int32), ("pending", C.c_int32), ("max_active", C.c_int32), ("reserved", C.c_int32)]


class sw_ms_block_header(C.Structure):
    _fields_ = [("project", C.c_char_p), ("system", C.c_char_p), ("fasta", C.c_char_p),
                ("rank", C.c_int32), ("row_block", C.c_int32), ("col_block", C.c_int32),
                ("row_start", C.c_int32), ("row_end", C.c_int32), ("col_start", C.c_int32),
                ("col_end", C.c_int32), ("row_start_id", C.c_char_p), ("row_end_id", C.c_char_p),
                ("col_start_id", C.c_char_p), ("col_end_id", C.c_char_p)]


_lib = None
P = C.c_void_p
I32, I64 = C.c_int32, C.c_int64


def load():
    """The loaded library; raises when it has not been built (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `python -m csharp_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    sig = {
        "sw_create": ([C.POINTER(sw_config), C.POINTER(P)], I32),
        "sw_destroy": ([P], I32),
        "sw_last_error": ([P], C.c_char_p),
        "sw_version": ([], C.c_char_p),
        "sw_upload_sequences": ([P, P, P, I32], I32),
        "sw_compute_block": ([P, I32, I32, I32, I32, I32, P, I64, C.POINTER(I64)], I32),
        "sw_compute_block_device": ([P, I32, I32, I32, I32, I32, P, I64, C.POINTER(I64)], I32),
        "sw_align_pair": ([P, P, I32, P, I32, C.POINTER(sw_pair_result)], I32),
        "sw_all_pairs_device": ([P, I32, P, I64, C.POINTER(I64), C.POINTER(I64)], I32),
        "sw_all_pairs": ([P, I32, P, I64, C.POINTER(I64), C.POINTER(I64)], I32),
        "sw_last_rerun_count": ([P, C.POINTER(I64)], I32),
        "sw_synchronize": ([P], I32),
        "sw_parse_scoring_matrix": ([C.c_char_p, I64, P], I32),
        "sw_builtin_scoring_matrix": ([C.c_char_p, P], I32),
        "sw_parse_fasta": ([C.c_char_p, I64, P, P, C.POINTER(I32), C.POINTER(I64)], I32),
        "sw_partition_ranges": ([I32, I32, I32, P, P], I32),
        "sw_block_is_computed": ([I32, I32], I32),
        "sw_write_full_matrix": ([C.c_char_p, P, I64, I64, I64], I32),
        "sw_write_ms_block": ([C.c_char_p, C.POINTER(sw_ms_block_header), P, I64], I32),
        "sw_read_ms_block_dims": ([C.c_char_p] + [C.POINTER(I32)] * 7, I32),
        "sw_read_ms_block_values": ([C.c_char_p, P, I64], I32),
        "sw_measure_int_peak": ([I32, C.POINTER(C.c_double), C.POINTER(C.c_double)], I32),
        "sw_set_option": ([P, C.c_char_p, I64], I32),
        "sw_compute_rank_blocks": ([P, I32, I32, P, I64, C.POINTER(I64)], I32),
        "sw_compute_rows": ([P, I32, I32, P, I64, C.POINTER(I64)], I32),
        "sw_query": ([P, C.c_char_p, C.POINTER(I64)], I32),
        "sw_compute_block_static": ([C.POINTER(sw_config), P, P, I32, I32, I32, I32, I32, I32, P, I64,
                                     C.POINTER(I64), P], I32),
        "sw_submit_job": ([P, P, P, I32, P, I64, C.POINTER(I64)], I32),
        "sw_poll": ([P, I64, I32, C.POINTER(I32), C.POINTER(sw_job_info)], I32),
        "sw_serve_stats": ([P, C.POINTER(sw_serve_counters)], I32),
        "sw_serve_drain": ([P], I32),
        "sw_autotune": ([P, P, I64, P], I32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(status, ctx=None):
    if status != SW_OK:
        msg = load().sw_last_error(ctx).decode() if ctx else ""
        raise SwError(status, msg)


def ptr(a: np.ndarray):
    return a.ctypes.data_as(P)
