"""The scoring server: guide-set requests admitted by device-memory footprint and scored with
continuous batching over several in-flight slots (Python face of issl_server_* in
include/issl_b200.h)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import RequestInfo, ServerConfig, ServerSummary, check, lib
from .index import Index, ScoreResult, _method, _u64

STATUS_TIMEOUT = -6


@dataclass
class Reply:
    result: ScoreResult
    info: RequestInfo


class Server:
    """Requests are submitted from any thread and collected with wait(); the native slots score
    them in the background."""

    def __init__(self, index: Index, n_slots: int = 0, max_batch_guides: int = 0, headroom_bytes: int = 0,
                 max_wait_us: int = 0):
        self.index = index
        cfg = ServerConfig(n_slots, max_wait_us, max_batch_guides, headroom_bytes)
        h = C.c_void_p()
        check(lib().issl_server_create(index.handle, C.byref(cfg), C.byref(h)))
        self._h = h
        self._sizes = {}

    def close(self) -> None:
        if self._h and self._h.value:
            lib().issl_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, sigs, method="and", threshold: float = 75.0, max_dist: int = 4) -> int:
        s = np.ascontiguousarray(sigs, dtype=np.uint64)
        t = C.c_uint64()
        check(lib().issl_server_submit(self._h, _u64(s), len(s), _method(method), threshold, max_dist, C.byref(t)))
        self._sizes[t.value] = len(s)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """The request's results and timing; None if it is not finished within timeout_ms."""
        n = self._sizes[ticket]
        mit = np.zeros(n, np.float64)
        cfd = np.zeros(n, np.float64)
        code = C.create_string_buffer(max(n, 1))
        cnt = np.zeros(n, np.uint64)
        info = RequestInfo()
        f = C.POINTER(C.c_double)
        rc = lib().issl_server_wait(self._h, ticket, timeout_ms, mit.ctypes.data_as(f), cfd.ctypes.data_as(f), code,
                                    _u64(cnt), C.byref(info))
        if rc == STATUS_TIMEOUT:
            return None
        del self._sizes[ticket]
        check(rc)
        return Reply(ScoreResult(mit, cfd, code.raw[:n], cnt, None), info)

    def stats(self, reset: bool = False) -> ServerSummary:
        out = ServerSummary()
        check(lib().issl_server_stats(self._h, C.byref(out), int(reset)))
        return out
