"""ctypes binding of libscb_b200.so (the C ABI in include/scb.h).

There is no CPU fallback: if the shared library is missing, loading raises; if no CUDA device
is present, every compute entry point returns SCB_ERR_INTERNAL_STATE, which the Python layer
raises as InternalState.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libscb_b200.so")
HEADER = os.path.join(ROOT, "include", "scb.h")

SCB_OK = 0
STRATEGIES = {"auto": 0, "plain": 1, "fused": 2, "staged": 3, "grouped": 4}


class ScbConfig(C.Structure):
    _fields_ = [
        ("k", C.c_uint64), ("m", C.c_uint64), ("s", C.c_uint64), ("n_hashes", C.c_uint64),
        ("counter_bits", C.c_uint8), ("counter_slots_exponent", C.c_uint8),
        ("block_slots_exponent", C.c_uint8), ("threads", C.c_uint64), ("queue", C.c_uint64),
    ]


class ScbReport(C.Structure):
    _fields_ = [
        ("records_processed", C.c_uint64), ("total_windows", C.c_uint64), ("valid_kmers", C.c_uint64),
        ("positive_estimates", C.c_uint64), ("estimate_checksum", C.c_uint64),
    ]


class ScbStats(C.Structure):
    _fields_ = [("windows", C.c_uint64), ("super_kmers", C.c_uint64), ("smers", C.c_uint64),
                ("sectors", C.c_uint64)]


class ScbTimings(C.Structure):
    _fields_ = [("pack_ms", C.c_double), ("insert_ms", C.c_double), ("query_ms", C.c_double),
                ("batches", C.c_uint64), ("cut_ms", C.c_double), ("bucket_ms", C.c_double),
                ("apply_insert_ms", C.c_double), ("apply_query_ms", C.c_double)]


class ScbServerConfig(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_uint64), ("max_batch_bytes", C.c_uint64),
                ("max_batch_seqs", C.c_uint64), ("max_inflight", C.c_uint32), ("reserved", C.c_uint32),
                ("spectrum_keys", C.c_uint64)]


class ScbRequestStats(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("service_ms", C.c_double), ("total_ms", C.c_double),
                ("windows", C.c_uint64)]


class ScbServerSummary(C.Structure):
    _fields_ = [("requests", C.c_uint64), ("windows", C.c_uint64), ("batches", C.c_uint64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
                ("span_s", C.c_double), ("slots", C.c_uint32), ("reserved", C.c_uint32)]


class ScbTuning(C.Structure):
    _fields_ = [("small_batch_bytes", C.c_uint64), ("insert_small", C.c_int32), ("insert_large", C.c_int32),
                ("query_small", C.c_int32), ("query_large", C.c_int32), ("bucket_records", C.c_uint32),
                ("apply_threads", C.c_uint32), ("host_batch_bytes", C.c_uint64), ("insert_ms", C.c_double),
                ("query_ms", C.c_double), ("candidates", C.c_uint32), ("reserved", C.c_uint32)]

    def as_dict(self) -> dict:
        names = {v: k for k, v in STRATEGIES.items()}
        return {"small_batch_bytes": self.small_batch_bytes, "insert_small": names.get(self.insert_small),
                "insert_large": names.get(self.insert_large), "query_small": names.get(self.query_small),
                "query_large": names.get(self.query_large), "bucket_records": self.bucket_records,
                "apply_threads": self.apply_threads, "host_batch_bytes": self.host_batch_bytes,
                "sample_insert_ms": self.insert_ms, "sample_query_ms": self.query_ms,
                "candidates": self.candidates}


_lib = None


def declared_symbols() -> list[str]:
    """Function names declared in include/scb.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(scb_[a-z0-9_]+)\s*\(", text)))


def load(path: str | None = None):
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or os.environ.get("SCB_B200_LIB", LIB_PATH)
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: build it with `python -m scbf_b200.build` "
                           "(the CUDA library has no CPU fallback)")
    L = C.CDLL(p)
    vp, u8p, u32p, u64p = C.c_void_p, C.POINTER(C.c_uint8), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
    ctxp = C.c_void_p
    sig = {
        "scb_last_error": (C.c_char_p, []),
        "scb_version": (C.c_char_p, []),
        "scb_kernel_launches": (C.c_uint64, []),
        "scb_config_default": (C.c_int, [C.POINTER(ScbConfig)]),
        "scb_config_validate": (C.c_int, [C.POINTER(ScbConfig)]),
        "scb_create": (C.c_int, [C.POINTER(ScbConfig), C.POINTER(ctxp)]),
        "scb_destroy": (None, [ctxp]),
        "scb_insert_batch": (C.c_int, [ctxp, vp, vp, C.c_uint64, u64p, u64p]),
        "scb_insert_batch_device": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.c_uint64, vp, u64p, u64p]),
        "scb_freeze": (C.c_int, [ctxp]),
        "scb_get_counts": (C.c_int, [ctxp, u64p, u64p]),
        "scb_get_config": (C.c_int, [ctxp, C.POINTER(ScbConfig)]),
        "scb_set_threads": (C.c_int, [ctxp, C.c_uint64]),
        "scb_query_batch": (C.c_int, [ctxp, vp, vp, C.c_uint64, vp, vp]),
        "scb_query_batch_device": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.c_uint64, vp, vp, vp]),
        "scb_count_windows": (C.c_uint64, [ctxp, vp, C.c_uint64]),
        "scb_records_indexed": (C.c_uint64, [ctxp, vp, vp, C.c_uint64]),
        "scb_query_report": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.POINTER(ScbReport)]),
        "scb_query_report_device": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.c_uint64, vp, C.POINTER(ScbReport)]),
        "scb_build_and_stream_query": (C.c_int, [ctxp, vp, vp, C.c_uint64, u64p, u64p, C.POINTER(ScbReport)]),
        "scb_build_and_stream_query_device": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.c_uint64, vp, u64p, u64p,
                                                        C.POINTER(ScbReport)]),
        "scb_spectrum_distinct": (C.c_int, [ctxp, vp, vp, C.c_uint64, vp, vp, C.c_uint64, u64p, u64p, u64p]),
        "scb_counter_histogram": (C.c_int, [ctxp, vp, vp, C.c_uint64, u64p]),
        "scb_save": (C.c_int, [ctxp, C.c_char_p]),
        "scb_load": (C.c_int, [C.c_char_p, C.POINTER(ctxp)]),
        "scb_table_bytes": (C.c_uint64, [ctxp]),
        "scb_table_download": (C.c_int, [ctxp, vp, C.c_uint64]),
        "scb_table_download_range": (C.c_int, [ctxp, C.c_uint64, vp, C.c_uint64]),
        "scb_table_upload": (C.c_int, [ctxp, vp, C.c_uint64, C.c_uint64]),
        "scb_set_strategy": (C.c_int, [ctxp, C.c_int, C.c_int]),
        "scb_get_strategy": (C.c_int, [ctxp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "scb_batch_stats": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.POINTER(ScbStats)]),
        "scb_debug_window_minimizers": (C.c_int, [ctxp, vp, vp, C.c_uint64, vp]),
        "scb_set_timing": (C.c_int, [ctxp, C.c_int]),
        "scb_get_timings": (C.c_int, [ctxp, C.POINTER(ScbTimings)]),
        "scb_set_graphs": (C.c_int, [ctxp, C.c_int]),
        "scb_set_piece_bytes": (C.c_int, [ctxp, C.c_uint64]),
        "scb_set_host_pack": (C.c_int, [ctxp, C.c_int]),
        "scb_h2d_bytes": (C.c_int, [ctxp, C.POINTER(C.c_uint64)]),
        "scb_set_fused_build": (C.c_int, [ctxp, C.c_int]),
        "scb_fastx_read": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
        "scb_fastx_sequences": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), u64p]),
        "scb_fastx_headers": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp)]),
        "scb_fastx_free": (None, [vp]),
        "scb_graph_stats": (C.c_int, [ctxp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "scb_reset": (C.c_int, [ctxp]),
        "scb_query_report_device_noalloc": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.c_uint64, vp,
                                                      C.POINTER(ScbReport)]),
        "scb_server_create": (C.c_int, [ctxp, C.POINTER(ScbServerConfig), C.POINTER(vp)]),
        "scb_server_submit": (C.c_int, [vp, vp, vp, C.c_uint64, vp, vp, u64p]),
        "scb_server_wait": (C.c_int, [vp, C.c_uint64, C.POINTER(ScbRequestStats)]),
        "scb_server_get_summary": (C.c_int, [vp, C.POINTER(ScbServerSummary)]),
        "scb_server_reset_stats": (C.c_int, [vp]),
        "scb_server_graph_stats": (C.c_int, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "scb_server_spectrum": (C.c_int, [vp, vp, vp, C.c_uint64, u64p, u64p, u64p]),
        "scb_server_destroy": (None, [vp]),
        "scb_autotune": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.POINTER(ScbTuning)]),
        "scb_get_tuning": (C.c_int, [ctxp, C.POINTER(ScbTuning)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return (load().scb_last_error() or b"").decode(errors="replace")
