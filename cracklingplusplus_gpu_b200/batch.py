"""Batched scoring: many guide sets, each with its own method / threshold / max_dist, in one
graph-captured pass (Python face of the issl_batch_* entry points of include/issl_b200.h)."""
from __future__ import annotations

import ctypes as C
from typing import Sequence, Tuple

import numpy as np

from ._lib import GuideSet, ScoreStats, check, lib
from .index import Index, ScoreResult, _method, _u64

SetSpec = Tuple[int, object, float, int]  # (count, method, threshold, max_dist)


def set_table(sets: Sequence[SetSpec]):
    arr = (GuideSet * max(len(sets), 1))()
    for i, (count, method, threshold, max_dist) in enumerate(sets):
        arr[i] = GuideSet(int(count), _method(method), int(max_dist), float(threshold))
    return arr


class Batch:
    """A batch context on the index's GPU: its own workspace and captured graph. Not
    thread-safe; use one per thread."""

    def __init__(self, index: Index):
        self.index = index
        h = C.c_void_p()
        check(lib().issl_batch_create(index.handle, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h and self._h.value:
            lib().issl_batch_destroy(self._h)
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

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def score(self, sigs, sets: Sequence[SetSpec]) -> ScoreResult:
        """sigs: uint64 signatures of all guides, set after set; sets: (count, method,
        threshold, max_dist) per set. Returns per-guide results (distinct is None)."""
        s = np.ascontiguousarray(sigs, dtype=np.uint64)
        n = len(s)
        tab = set_table(sets)
        mit = np.zeros(n, np.float64)
        cfd = np.zeros(n, np.float64)
        code = C.create_string_buffer(max(n, 1))
        cnt = np.zeros(n, np.uint64)
        f = C.POINTER(C.c_double)
        check(lib().issl_batch_score_host(self._h, _u64(s), n, tab, len(sets), mit.ctypes.data_as(f),
                                          cfd.ctypes.data_as(f), code, _u64(cnt)))
        return ScoreResult(mit, cfd, code.raw[:n], cnt, None)

    def score_device(self, d_sigs: int, n: int, sets: Sequence[SetSpec], d_mit: int, d_cfd: int, d_code: int,
                     d_count: int = 0, stream: int = 0) -> None:
        tab = set_table(sets)
        check(lib().issl_batch_score(self._h, C.c_void_p(d_sigs), n, tab, len(sets), C.c_void_p(d_mit or None),
                                     C.c_void_p(d_cfd or None), C.c_void_p(d_code), C.c_void_p(d_count or None),
                                     C.c_void_p(stream or None)))

    def stats(self) -> ScoreStats:
        out = ScoreStats()
        check(lib().issl_batch_stats(self._h, C.byref(out)))
        return out
