"""ctypes bindings of libissl_b200.so (the C ABI of include/issl_b200.h and issl_b200_module.hpp)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_NAME = "libissl_b200.so"

# otScoreMethod, include/util.hpp:20 (and the INI names of lib/util.cpp:13-19)
OT_METHODS = {"mit": 0, "cfd": 1, "mitAndCfd": 2, "mitOrCfd": 3, "avgMitCfd": 4}
# method words of the ISSLScoreOfftargets command line (ISSLScoreOfftargets.cpp:69-91)
CLI_METHODS = {"mit": 0, "cfd": 1, "and": 2, "or": 3, "avg": 4}

STATUS = {0: "ok", -1: "invalid argument", -2: "I/O error", -3: "format error", -4: "out of memory",
          -5: "CUDA error", -6: "timeout", -7: "unsupported", -8: "busy",
          -9: "internal consistency check failed"}


class IsslError(RuntimeError):
    """A failing library call: .code is the ISSL_ERR_* status, str() the library's message."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} [{STATUS.get(code, code)}]")
        self.code = code


class IndexInfo(C.Structure):
    _fields_ = [("n_sites", C.c_uint64), ("seq_len", C.c_uint64), ("n_slices", C.c_uint64),
                ("n_buckets", C.c_uint64), ("device_bytes", C.c_uint64), ("device", C.c_int),
                ("min_width", C.c_int), ("max_width", C.c_int), ("entry_bytes", C.c_int),
                ("host_bytes", C.c_uint64), ("window_slices", C.c_int)]


class ScoreStats(C.Structure):
    _fields_ = [("scan_ms", C.c_double), ("total_ms", C.c_double), ("probes", C.c_uint64),
                ("buckets_scanned", C.c_uint64), ("entries_scanned", C.c_uint64), ("units", C.c_uint64),
                ("hits", C.c_uint64), ("scan_bytes", C.c_uint64), ("launches", C.c_uint64),
                ("class_probes", C.c_uint64 * 3), ("candidates", C.c_uint64), ("staged_bytes", C.c_uint64),
                ("dropped_hits", C.c_uint64), ("replayed", C.c_uint64), ("runs", C.c_uint64)]


class Tuning(C.Structure):
    """issl_tuning: scan unit size per bucket-size class (<64, 64..4095, >=4096 entries),
    staging depth, scan blocks per SM (0 = as many as fit), slices of the first wave."""
    _fields_ = [("chunk", C.c_uint32 * 3), ("stages", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("first_wave", C.c_uint32)]

    def as_tuple(self):
        return (tuple(self.chunk), self.stages, self.blocks_per_sm, self.first_wave)


class TuneReport(C.Structure):
    _fields_ = [("default_ms", C.c_double), ("best_ms", C.c_double), ("configs_timed", C.c_uint32),
                ("from_cache", C.c_uint32), ("class_probes", C.c_uint64 * 3)]


class ServerConfig(C.Structure):
    """issl_server_config (zeros select the defaults: 3 slots, 131072 guides per batch, 16 GiB headroom)."""
    _fields_ = [("n_slots", C.c_uint32), ("max_wait_us", C.c_uint32), ("max_batch_guides", C.c_uint64),
                ("headroom_bytes", C.c_uint64)]


class RequestInfo(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("service_ms", C.c_double), ("latency_ms", C.c_double),
                ("batch_guides", C.c_uint64), ("batch_requests", C.c_uint32), ("slot", C.c_uint32)]


class ServerSummary(C.Structure):
    _fields_ = [("requests", C.c_uint64), ("guides", C.c_uint64), ("batches", C.c_uint64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("max_ms", C.c_double), ("mean_batch_guides", C.c_double),
                ("slots", C.c_uint32), ("peak_in_flight", C.c_uint32), ("slot_budget_bytes", C.c_uint64),
                ("peak_batch_bytes", C.c_uint64)]


class GuideSet(C.Structure):
    """issl_guide_set: one set of a batch (consecutive guides sharing method/threshold/max_dist)."""
    _fields_ = [("count", C.c_uint64), ("method", C.c_int), ("max_dist", C.c_int), ("threshold", C.c_double)]


class SynthSpecC(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_sites", C.c_uint64), ("repeat_frac", C.c_double),
                ("n_repeat_seeds", C.c_uint64), ("repeat_lambda", C.c_double), ("n_queries", C.c_uint64),
                ("copied_frac", C.c_double), ("repeat_query_frac", C.c_double), ("planted_into_sites", C.c_int),
                ("slice_masks", C.POINTER(C.c_uint64)), ("n_slices", C.c_uint64)]


def library_path() -> str:
    return os.path.join(HERE, _LIB_NAME)


_lib = None

P = C.POINTER
u64p = P(C.c_uint64)
f64p = P(C.c_double)
vp = C.c_void_p

# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("issl_last_error", C.c_char_p, []),
    ("issl_open", C.c_int, [C.c_char_p, C.c_int, P(vp)]),
    ("issl_open_mapped", C.c_int, [C.c_char_p, C.c_int, C.c_uint32, P(vp)]),
    ("issl_index_set_list_placement", C.c_int, [vp, C.c_uint32]),
    ("issl_open_arrays", C.c_int, [u64p, C.c_uint64, C.c_uint64, u64p, C.c_uint64, u64p, u64p, C.c_int, P(vp)]),
    ("issl_build", C.c_int, [u64p, P(C.c_uint32), C.c_uint64, u64p, C.c_uint64, C.c_int, P(vp)]),
    ("issl_close", C.c_int, [vp]),
    ("issl_index_get_info", C.c_int, [vp, P(IndexInfo)]),
    ("issl_export", C.c_int, [vp, u64p, u64p, u64p, u64p]),
    ("issl_save", C.c_int, [vp, C.c_char_p]),
    ("issl_score", C.c_int, [vp, C.c_char_p, C.c_size_t, C.c_size_t, C.c_int, C.c_double, C.c_int, f64p, f64p,
                             C.c_char_p, u64p, u64p]),
    ("issl_score_sigs", C.c_int, [vp, u64p, C.c_size_t, C.c_int, C.c_double, C.c_int, f64p, f64p, C.c_char_p,
                                  u64p, u64p]),
    ("issl_score_device", C.c_int, [vp, vp, C.c_size_t, C.c_int, C.c_double, C.c_int, vp, vp, vp, vp, vp, vp]),
    ("issl_score_device_static", C.c_int, [vp, vp, C.c_size_t, C.c_int, C.c_double, C.c_int, vp, vp, vp, vp, vp]),
    ("issl_last_stats", C.c_int, [vp, P(ScoreStats)]),
    ("issl_get_tuning", C.c_int, [vp, P(Tuning)]),
    ("issl_set_tuning", C.c_int, [vp, P(Tuning)]),
    ("issl_autotune", C.c_int, [vp, vp, C.c_size_t, C.c_int, C.c_double, C.c_int, C.c_char_p, P(Tuning),
                                P(TuneReport)]),
    ("issl_batch_create", C.c_int, [vp, P(vp)]),
    ("issl_batch_destroy", None, [vp]),
    ("issl_batch_score", C.c_int, [vp, vp, C.c_size_t, P(GuideSet), C.c_size_t, vp, vp, vp, vp, vp]),
    ("issl_batch_score_host", C.c_int, [vp, u64p, C.c_size_t, P(GuideSet), C.c_size_t, f64p, f64p, C.c_char_p,
                                        u64p]),
    ("issl_batch_stats", C.c_int, [vp, P(ScoreStats)]),
    ("issl_workspace_bytes", C.c_int, [vp, C.c_uint64, C.c_double, u64p]),
    ("issl_index_trim", C.c_int, [vp]),
    ("issl_extract_offtargets", C.c_int, [P(C.c_char_p), C.c_size_t, C.c_char_p, C.c_int, u64p]),
    ("issl_build_from_sequences", C.c_int, [P(C.c_char_p), C.c_size_t, u64p, C.c_uint64, C.c_int, P(vp), u64p]),
    ("issl_server_create", C.c_int, [vp, P(ServerConfig), P(vp)]),
    ("issl_server_submit", C.c_int, [vp, u64p, C.c_size_t, C.c_int, C.c_double, C.c_int, u64p]),
    ("issl_server_wait", C.c_int, [vp, C.c_uint64, C.c_int, f64p, f64p, C.c_char_p, u64p, P(RequestInfo)]),
    ("issl_server_stats", C.c_int, [vp, P(ServerSummary), C.c_int]),
    ("issl_server_destroy", None, [vp]),
    ("issl_synth", C.c_int, [P(SynthSpecC), C.c_int, P(vp), u64p]),
    ("issl_tables", C.c_int, [u64p, f64p, f64p, f64p]),
    ("issl_module_run", C.c_int, [C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_size_t,
                                  C.c_char_p, C.c_size_t, P(C.c_uint8), P(C.c_int8), C.c_char_p, f64p, f64p,
                                  C.c_char_p]),
    ("issl_module_release_all", C.c_int, []),
    ("issl_module_open", C.c_int, [C.c_char_p, C.c_int, C.c_int, P(vp)]),
]


def lib():
    """The loaded native library; raises ImportError when it has not been built."""
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise ImportError(
                f"{path} is missing: build the CUDA library first "
                "(python -m cracklingplusplus_gpu_b200.build); there is no CPU fallback")
        L = C.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        msg = lib().issl_last_error()
        raise IsslError(rc, msg.decode(errors="replace") if msg else "error")
