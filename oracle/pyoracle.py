"""ctypes wrapper around oracle/liboracle.so -- the CPU checker (test infrastructure only).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

METHODS = {"mit": 0, "cfd": 1, "mitAndCfd": 2, "mitOrCfd": 3, "avgMitCfd": 4}
CLI_METHODS = {"mit": 0, "cfd": 1, "and": 2, "or": 3, "avg": 4}


class OraIndex(C.Structure):
    _fields_ = [
        ("n_sites", C.c_uint64),
        ("seq_len", C.c_uint64),
        ("n_slices", C.c_uint64),
        ("sigs", C.POINTER(C.c_uint64)),
        ("slice_masks", C.POINTER(C.c_uint64)),
        ("list_sizes", C.POINTER(C.c_uint64)),
        ("lists", C.POINTER(C.c_uint64)),
        ("owns_memory", C.c_int),
    ]


def build_lib() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_lib()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.ora_encode.restype = C.c_uint64
        L.ora_encode.argtypes = [C.c_char_p, C.c_uint64]
        L.ora_mit_table.argtypes = [P(C.c_uint64), P(C.c_double)]
        L.ora_set_cfd_tables.argtypes = [P(C.c_double), P(C.c_double)]
        L.ora_load.argtypes = [C.c_char_p, P(OraIndex)]
        L.ora_free.argtypes = [P(OraIndex)]
        L.ora_build.argtypes = [P(C.c_uint64), P(C.c_uint32), C.c_uint64, P(C.c_uint64), C.c_uint64,
                                C.c_uint64, P(OraIndex)]
        L.ora_write.argtypes = [C.c_char_p, P(OraIndex)]
        L.ora_score.argtypes = [P(OraIndex), P(C.c_uint64), C.c_uint64, C.c_int, C.c_double, C.c_int,
                                C.c_int, P(C.c_double), P(C.c_double), P(C.c_uint64), P(C.c_uint64)]
        L.ora_finalise.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, P(C.c_double),
                                   P(C.c_double), C.c_char_p]
        L.ora_bruteforce.argtypes = [P(C.c_uint64), P(C.c_uint32), C.c_uint64, P(C.c_uint64), C.c_uint64,
                                     C.c_int, C.c_int, P(C.c_double), P(C.c_double), P(C.c_uint64)]
        L.ora_synth.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_uint64, C.c_double, C.c_uint64, C.c_double,
                                C.c_double, C.c_int, P(C.c_uint64), P(C.c_uint32), P(C.c_uint64)]
        L.ora_write_built.argtypes = [C.c_char_p, P(C.c_uint64), P(C.c_uint32), C.c_uint64, P(C.c_uint64),
                                      C.c_uint64]
        L.ora_trace.restype = C.c_uint64
        L.ora_trace.argtypes = [C.POINTER(OraIndex), C.c_uint64, C.c_int, P(C.c_double), P(C.c_double),
                                P(C.c_uint32), C.c_uint64]
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def set_cfd_tables(pos320, pam16) -> None:
    pos = np.ascontiguousarray(pos320, dtype=np.float64)
    pam = np.ascontiguousarray(pam16, dtype=np.float64)
    assert pos.size == 320 and pam.size == 16
    lib().ora_set_cfd_tables(_p(pos, C.c_double), _p(pam, C.c_double))


def mit_table():
    n = lib().ora_mit_table(None, None)
    masks = np.zeros(n, np.uint64)
    vals = np.zeros(n, np.float64)
    lib().ora_mit_table(_p(masks, C.c_uint64), _p(vals, C.c_double))
    return masks, vals


def encode(seq: str) -> int:
    return int(lib().ora_encode(seq.encode(), 20))


class Index:
    """A reference-layout index held by the oracle."""

    def __init__(self):
        self.s = OraIndex()
        self._keep = []

    @classmethod
    def load(cls, path: str) -> "Index":
        ix = cls()
        rc = lib().ora_load(path.encode(), C.byref(ix.s))
        if rc != 0:
            raise RuntimeError(f"oracle: cannot load {path} (rc={rc})")
        return ix

    @classmethod
    def build(cls, sigs, occ, masks, seq_len: int = 20) -> "Index":
        ix = cls()
        sigs = np.ascontiguousarray(sigs, np.uint64)
        occ = np.ascontiguousarray(occ, np.uint32)
        masks = np.ascontiguousarray(masks, np.uint64)
        lib().ora_build(_p(sigs, C.c_uint64), _p(occ, C.c_uint32), len(sigs), _p(masks, C.c_uint64),
                        len(masks), seq_len, C.byref(ix.s))
        return ix

    @classmethod
    def from_arrays(cls, sigs, masks, list_sizes, lists, seq_len: int = 20) -> "Index":
        """Wrap arrays already in the reference layout (no copy; arrays kept alive)."""
        ix = cls()
        arrs = [np.ascontiguousarray(a, np.uint64) for a in (sigs, masks, list_sizes, lists)]
        ix._keep = arrs
        ix.s.n_sites = len(arrs[0])
        ix.s.seq_len = seq_len
        ix.s.n_slices = len(arrs[1])
        ix.s.sigs, ix.s.slice_masks, ix.s.list_sizes, ix.s.lists = (_p(a, C.c_uint64) for a in arrs)
        ix.s.owns_memory = 0
        return ix

    def write(self, path: str) -> None:
        rc = lib().ora_write(path.encode(), C.byref(self.s))
        if rc != 0:
            raise RuntimeError(f"oracle: cannot write {path}")

    def arrays(self):
        n, S = self.s.n_sites, self.s.n_slices
        sigs = np.ctypeslib.as_array(self.s.sigs, (n,)).copy() if n else np.zeros(0, np.uint64)
        masks = np.ctypeslib.as_array(self.s.slice_masks, (S,)).copy()
        total = sum(1 << (2 * bin(int(m) & ((1 << self.s.seq_len) - 1)).count("1")) for m in masks)
        sizes = np.ctypeslib.as_array(self.s.list_sizes, (total,)).copy()
        lists = np.ctypeslib.as_array(self.s.lists, (n * S,)).copy() if n else np.zeros(0, np.uint64)
        return sigs, masks, sizes, lists

    def score(self, qsigs, method: int, threshold: float, max_dist: int = 4, threads: int = 0):
        q = np.ascontiguousarray(qsigs, np.uint64)
        nq = len(q)
        mit = np.zeros(nq, np.float64)
        cfd = np.zeros(nq, np.float64)
        cnt = np.zeros(nq, np.uint64)
        distinct = np.zeros(1, np.uint64)
        rc = lib().ora_score(C.byref(self.s), _p(q, C.c_uint64), nq, method, threshold, max_dist, threads,
                             _p(mit, C.c_double), _p(cfd, C.c_double), _p(cnt, C.c_uint64),
                             _p(distinct, C.c_uint64))
        if rc != 0:
            raise RuntimeError("oracle: MIT table lookup failed (the reference would throw)")
        return mit, cfd, cnt, int(distinct[0])

    def trace(self, qsig: int, max_dist: int = 4):
        """The scored terms of one guide in the reference's adding order, no early exit:
        (mit_terms, cfd_terms, occurrences) arrays."""
        n = int(lib().ora_trace(C.byref(self.s), int(qsig), max_dist, None, None, None, 0))
        mit = np.zeros(max(n, 1))
        cfd = np.zeros(max(n, 1))
        occ = np.zeros(max(n, 1), np.uint32)
        lib().ora_trace(C.byref(self.s), int(qsig), max_dist, _p(mit, C.c_double), _p(cfd, C.c_double),
                        _p(occ, C.c_uint32), n)
        return mit[:n], cfd[:n], occ[:n]

    def free(self):
        if self.s.owns_memory:
            lib().ora_free(C.byref(self.s))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def synth(seed: int, n_sites: int, n_queries: int, repeat_frac: float = 0.05, n_repeat_seeds: int = 10000,
          repeat_lambda: float = 2.0, copied_frac: float = 0.5, repeat_query_frac: float = 0.0,
          planted_into_sites: bool = False, threads: int = 0):
    """The library's seeded synthetic workload (issl_synth's spec), generated on the host:
    (sites uint64[n_sites], occ uint32[n_sites], queries uint64[n_queries])."""
    sites = np.zeros(n_sites, np.uint64)
    occ = np.zeros(n_sites, np.uint32)
    q = np.zeros(max(n_queries, 1), np.uint64)
    rc = lib().ora_synth(seed, n_sites, repeat_frac, n_repeat_seeds, repeat_lambda, n_queries, copied_frac,
                         repeat_query_frac, int(planted_into_sites), _p(sites, C.c_uint64), _p(occ, C.c_uint32),
                         _p(q, C.c_uint64))
    if rc != 0:
        raise RuntimeError(f"oracle synth failed (rc={rc})")
    return sites, occ, q[:n_queries]


def write_built(path: str, sigs, occ, masks) -> None:
    """Writes the .issl file of the sites bucketed by the slice masks (reference builder layout)."""
    sigs = np.ascontiguousarray(sigs, np.uint64)
    occ = np.ascontiguousarray(occ, np.uint32)
    masks = np.ascontiguousarray(masks, np.uint64)
    rc = lib().ora_write_built(path.encode(), _p(sigs, C.c_uint64), _p(occ, C.c_uint32), len(sigs),
                               _p(masks, C.c_uint64), len(masks))
    if rc != 0:
        raise RuntimeError(f"oracle: cannot write {path}")


def finalise(method: int, threshold: float, tot_mit, tot_cfd):
    n = len(tot_mit)
    ms = np.zeros(n)
    cs = np.zeros(n)
    codes = bytearray(n)
    m = C.c_double()
    c = C.c_double()
    code = C.create_string_buffer(1)
    for i in range(n):
        lib().ora_finalise(method, threshold, float(tot_mit[i]), float(tot_cfd[i]), C.byref(m), C.byref(c), code)
        ms[i], cs[i], codes[i] = m.value, c.value, code.raw[0]
    return ms, cs, bytes(codes)


def bruteforce(sigs, occ, qsigs, max_dist: int = 4, threads: int = 0):
    sigs = np.ascontiguousarray(sigs, np.uint64)
    occ = np.ascontiguousarray(occ, np.uint32)
    q = np.ascontiguousarray(qsigs, np.uint64)
    nq = len(q)
    mit = np.zeros(nq)
    cfd = np.zeros(nq)
    cnt = np.zeros(nq, np.uint64)
    lib().ora_bruteforce(_p(sigs, C.c_uint64), _p(occ, C.c_uint32), len(sigs), _p(q, C.c_uint64), nq, max_dist,
                         threads, _p(mit, C.c_double), _p(cfd, C.c_double), _p(cnt, C.c_uint64))
    return mit, cfd, cnt
