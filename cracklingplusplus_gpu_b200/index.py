"""Resident ISSL index and scoring calls (Python face of include/issl_b200.h)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from ._lib import CLI_METHODS, OT_METHODS, IndexInfo, ScoreStats, SynthSpecC, TuneReport, Tuning, check, lib


def _u64(a) -> C.POINTER(C.c_uint64):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _method(method) -> int:
    if isinstance(method, str):
        if method in OT_METHODS:
            return OT_METHODS[method]
        if method in CLI_METHODS:
            return CLI_METHODS[method]
        raise ValueError(f"Scoring method is not valid: {method!r}")
    return int(method)


@dataclass
class ScoreResult:
    """Per-guide outputs: scores (-1 where the method does not compute one), accept codes
    (b'1' accepted / b'0' rejected), occurrence-weighted off-target counts, distinct sites."""
    mit: np.ndarray
    cfd: np.ndarray
    code: bytes
    count: np.ndarray
    distinct: Optional[int]


@dataclass
class SynthSpec:
    """Seeded synthetic workload (see issl_synth_spec in include/issl_b200.h)."""
    seed: int
    n_sites: int
    slice_config: str
    n_queries: int
    repeat_frac: float = 0.05
    n_repeat_seeds: int = 10000
    repeat_lambda: float = 2.0
    copied_frac: float = 0.5
    repeat_query_frac: float = 0.0
    planted_into_sites: bool = False


class Index:
    """An ISSL index held resident on one GPU."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    # ---- construction -------------------------------------------------------------------
    @classmethod
    def open(cls, path: str, device: int = 0) -> "Index":
        h = C.c_void_p()
        check(lib().issl_open(path.encode(), device, C.byref(h)))
        return cls(h.value)

    @classmethod
    def open_mapped(cls, path: str, device: int = 0, window_slices: int = 4) -> "Index":
        """An index whose lists stay in page-locked host memory, for indexes larger than HBM
        (the reference's memory-mapped module): every scoring call streams them to the device
        window_slices slices at a time. Results are identical to Index.open."""
        h = C.c_void_p()
        check(lib().issl_open_mapped(path.encode(), device, window_slices, C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, sigs, slice_masks, list_sizes, lists, seq_len: int = 20, device: int = 0) -> "Index":
        arrs = [np.ascontiguousarray(a, dtype=np.uint64) for a in (sigs, slice_masks, list_sizes, lists)]
        h = C.c_void_p()
        check(lib().issl_open_arrays(_u64(arrs[0]), len(arrs[0]), seq_len, _u64(arrs[1]), len(arrs[1]),
                                     _u64(arrs[2]), _u64(arrs[3]), device, C.byref(h)))
        return cls(h.value)

    @classmethod
    def build(cls, sigs, occ, slice_masks, device: int = 0) -> "Index":
        s = np.ascontiguousarray(sigs, dtype=np.uint64)
        o = np.ascontiguousarray(occ, dtype=np.uint32)
        m = np.ascontiguousarray(slice_masks, dtype=np.uint64)
        h = C.c_void_p()
        check(lib().issl_build(_u64(s), o.ctypes.data_as(C.POINTER(C.c_uint32)), len(s), _u64(m), len(m), device,
                               C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_sequences(cls, inputs, slice_masks, device: int = 0):
        """Extracts the off-target sites of FASTA / plain-text files or directories on the GPU
        and builds the index from them; returns (index, number of sites extracted)."""
        paths = [p.encode() for p in inputs]
        arr = (C.c_char_p * len(paths))(*paths)
        m = np.ascontiguousarray(slice_masks, dtype=np.uint64)
        h = C.c_void_p()
        n = C.c_uint64()
        check(lib().issl_build_from_sequences(arr, len(paths), _u64(m), len(m), device, C.byref(h), C.byref(n)))
        return cls(h.value), n.value

    @classmethod
    def synth(cls, spec: SynthSpec, device: int = 0):
        """Generates the workload on the device; returns (index, query signatures)."""
        from .slice_configs import slice_masks
        masks = np.array(slice_masks(spec.slice_config), dtype=np.uint64)
        c = SynthSpecC(spec.seed, spec.n_sites, spec.repeat_frac, spec.n_repeat_seeds, spec.repeat_lambda,
                       spec.n_queries, spec.copied_frac, spec.repeat_query_frac, int(spec.planted_into_sites),
                       _u64(masks), len(masks))
        q = np.zeros(max(spec.n_queries, 1), dtype=np.uint64)
        h = C.c_void_p()
        check(lib().issl_synth(C.byref(c), device, C.byref(h), _u64(q)))
        return cls(h.value), q[:spec.n_queries]

    # ---- lifetime / inspection -----------------------------------------------------------
    def close(self) -> None:
        if self._h and self._h.value:
            check(lib().issl_close(self._h))
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

    def info(self) -> IndexInfo:
        out = IndexInfo()
        check(lib().issl_index_get_info(self._h, C.byref(out)))
        return out

    def export(self):
        """(sigs, slice_masks, list_sizes, lists) in the reference's file layout."""
        inf = self.info()
        sigs = np.zeros(inf.n_sites, np.uint64)
        masks = np.zeros(inf.n_slices, np.uint64)
        sizes = np.zeros(inf.n_buckets, np.uint64)
        lists = np.zeros(inf.n_sites * inf.n_slices, np.uint64)
        check(lib().issl_export(self._h, _u64(sigs), _u64(masks), _u64(sizes), _u64(lists)))
        return sigs, masks, sizes, lists

    def save(self, path: str) -> None:
        check(lib().issl_save(self._h, path.encode()))

    def set_list_placement(self, window_slices: int) -> None:
        """window_slices > 0: move the lists to page-locked host memory, streamed per call that
        many slices at a time; 0: back to HBM. The index must be idle."""
        check(lib().issl_index_set_list_placement(self._h, window_slices))

    def trim(self) -> None:
        """Frees the index's own scoring workspace (re-created by the next scoring call)."""
        check(lib().issl_index_trim(self._h))

    def last_stats(self) -> ScoreStats:
        out = ScoreStats()
        check(lib().issl_last_stats(self._h, C.byref(out)))
        return out

    # ---- tuning -----------------------------------------------------------------------------
    def get_tuning(self) -> Tuning:
        out = Tuning()
        check(lib().issl_get_tuning(self._h, C.byref(out)))
        return out

    def set_tuning(self, chunk=(1024, 1024, 1024), stages: int = 2, blocks_per_sm: int = 0,
                   first_wave: int = 1) -> None:
        t = Tuning((C.c_uint32 * 3)(*chunk), stages, blocks_per_sm, first_wave)
        check(lib().issl_set_tuning(self._h, C.byref(t)))

    def autotune(self, d_sigs: int, n: int, method="and", threshold: float = 75.0, max_dist: int = 4,
                 cache_path: Optional[str] = None):
        """Sweeps the scan tuning on a device-resident sample; returns (Tuning, TuneReport)."""
        t, r = Tuning(), TuneReport()
        check(lib().issl_autotune(self._h, C.c_void_p(d_sigs), n, _method(method), threshold, max_dist,
                                  cache_path.encode() if cache_path else None, C.byref(t), C.byref(r)))
        return t, r

    # ---- scoring --------------------------------------------------------------------------
    def score(self, guides, method="and", threshold: float = 75.0, max_dist: int = 4,
              distinct: bool = True) -> ScoreResult:
        """Score guides given as strings (first 20 nt used), a bytes buffer of fixed 21-byte
        lines, or a uint64 signature array."""
        m = _method(method)
        if isinstance(guides, np.ndarray) and guides.dtype == np.uint64:
            return self._score_sigs(guides, m, threshold, max_dist, distinct)
        if isinstance(guides, (bytes, bytearray)):
            buf, stride = bytes(guides), 21
            n = len(buf) // stride
        else:
            seqs = list(guides)
            stride = 21
            n = len(seqs)
            buf = b"".join((s.encode() if isinstance(s, str) else bytes(s))[:20].ljust(20, b"\0") + b"\n"
                           for s in seqs)
        return self._run(lambda out: lib().issl_score(self._h, buf, stride, n, m, threshold, max_dist, *out),
                         n, distinct)

    def _score_sigs(self, sigs, m, threshold, max_dist, distinct):
        s = np.ascontiguousarray(sigs, dtype=np.uint64)
        return self._run(lambda out: lib().issl_score_sigs(self._h, _u64(s), len(s), m, threshold, max_dist, *out),
                         len(s), distinct)

    @staticmethod
    def _run(call, n, distinct) -> ScoreResult:
        mit = np.zeros(n, np.float64)
        cfd = np.zeros(n, np.float64)
        code = C.create_string_buffer(max(n, 1))
        cnt = np.zeros(n, np.uint64)
        d = np.zeros(1, np.uint64)
        check(call((mit.ctypes.data_as(C.POINTER(C.c_double)), cfd.ctypes.data_as(C.POINTER(C.c_double)), code,
                    _u64(cnt), _u64(d) if distinct else None)))
        return ScoreResult(mit, cfd, code.raw[:n], cnt, int(d[0]) if distinct else None)

    def score_device(self, d_sigs: int, n: int, method, threshold: float, max_dist: int,
                     d_mit: int, d_cfd: int, d_code: int, d_count: int = 0, d_distinct: int = 0,
                     stream: int = 0) -> None:
        """All buffers are device pointers (e.g. torch tensor data_ptr()) on the index's GPU."""
        check(lib().issl_score_device(self._h, C.c_void_p(d_sigs), n, _method(method), threshold, max_dist,
                                      C.c_void_p(d_mit or None), C.c_void_p(d_cfd or None), C.c_void_p(d_code),
                                      C.c_void_p(d_count or None), C.c_void_p(d_distinct or None),
                                      C.c_void_p(stream or None)))


def extract_offtargets(inputs, out_path: str, device: int = 0) -> int:
    """ExtractOfftargets on the GPU: writes every site of the inputs, sorted, one per line;
    returns the number of lines."""
    paths = [p.encode() for p in inputs]
    arr = (C.c_char_p * len(paths))(*paths)
    n = C.c_uint64()
    check(lib().issl_extract_offtargets(arr, len(paths), out_path.encode(), device, C.byref(n)))
    return n.value


def tables():
    """(MIT masks, MIT scores, CFD position penalties, CFD PAM penalties) held by the library."""
    masks = np.zeros(6195, np.uint64)
    scores = np.zeros(6195, np.float64)
    pos = np.zeros(320, np.float64)
    pam = np.zeros(16, np.float64)
    f = C.POINTER(C.c_double)
    check(lib().issl_tables(_u64(masks), scores.ctypes.data_as(f), pos.ctypes.data_as(f), pam.ctypes.data_as(f)))
    return masks, scores, pos, pam


def encode(seq: str) -> int:
    """sequenceToSignature(seq, 20): C=1 G=2 T=3, anything else 0, base j at bits 2j."""
    v = 0
    for j, c in enumerate(seq[:20]):
        v |= {"C": 1, "G": 2, "T": 3}.get(c, 0) << (2 * j)
    return v


def decode(sig: int) -> str:
    return "".join("ACGT"[(int(sig) >> (2 * j)) & 3] for j in range(20))


def pack_guides(seqs: Sequence[str]) -> bytes:
    return b"".join(s.encode()[:20].ljust(20, b"\0") + b"\n" for s in seqs)
