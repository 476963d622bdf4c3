"""Deterministic small synthetic ISSL workloads (test infrastructure).

Sites and queries follow the benchmark workload composition at test sizes:
  * sites: 20-nt, 2-bit packed with base j at bits 2j..2j+1 (A=0 C=1 G=2 T=3), i.i.d. with
    GC 41% (P(A)=P(T)=0.295, P(C)=P(G)=0.205), a fraction drawn as copies of repeat seeds
    with Poisson(lambda) substitutions, made distinct by keeping the first occurrence;
  * occurrence counts min(1 + Geometric(p=0.9), 255), Geometric counting failures;
  * queries: a share copied from the sites with 0-4 planted substitutions (the mutated
    copy is inserted into the site set, so every distance 0..4 occurs), the rest random.

Every random draw comes from a counter-based splitmix64 stream so the cases are
bit-identical on every numpy version and machine.
"""
from __future__ import annotations

import numpy as np

U64 = np.uint64
MASK64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser (Steele, Lea, Flood 2014) applied elementwise to uint64."""
    with np.errstate(over="ignore"):
        z = x + U64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> U64(30))) * U64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> U64(27))) * U64(0x94D049BB133111EB)
        return z ^ (z >> U64(31))


class Stream:
    """Counter-based stream: draw k of stream (seed, tag) is splitmix64(key + k)."""

    def __init__(self, seed: int, tag: int):
        base = splitmix64(np.array([(seed * 0x100000001B3 + tag * 0x9E3779B1) & MASK64], dtype=U64))[0]
        self.key = U64(base)
        self.pos = 0

    def u64(self, n: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            idx = np.arange(self.pos, self.pos + n, dtype=U64) * U64(0xD1B54A32D192ED03) + self.key
        self.pos += n
        return splitmix64(idx)

    def uniform(self, n: int) -> np.ndarray:
        return (self.u64(n) >> U64(11)).astype(np.float64) * (1.0 / (1 << 53))

    def below(self, n: int, bound: int) -> np.ndarray:
        return (self.uniform(n) * bound).astype(np.int64)


def gc41_bases(u: np.ndarray) -> np.ndarray:
    """Uniform [0,1) -> base code with P(A)=P(T)=0.295, P(C)=P(G)=0.205."""
    return np.searchsorted(np.array([0.295, 0.5, 0.705]), u, side="right").astype(np.uint64)


def pack(bases: np.ndarray) -> np.ndarray:
    """(n, 20) base codes -> uint64 signatures, base j at bits 2j..2j+1."""
    shifts = (np.arange(bases.shape[1], dtype=np.uint64) * U64(2))[None, :]
    return np.bitwise_or.reduce(bases.astype(np.uint64) << shifts, axis=1)


def random_sigs(st: Stream, n: int) -> np.ndarray:
    return pack(gc41_bases(st.uniform(n * 20)).reshape(n, 20))


def substitute(st: Stream, sigs: np.ndarray, n_subs: np.ndarray) -> np.ndarray:
    """Apply n_subs[i] substitutions at uniform distinct positions with a different base."""
    out = sigs.copy()
    for i in range(len(sigs)):
        k = int(n_subs[i])
        if k == 0:
            continue
        keys = st.u64(20)
        positions = np.argsort(keys, kind="stable")[:k]
        delta = 1 + st.below(k, 3)
        s = int(out[i])
        for p, d in zip(positions.tolist(), delta.tolist()):
            b = (s >> (2 * p)) & 3
            s = (s & ~(3 << (2 * p))) | (((b + d) & 3) << (2 * p))
        out[i] = s
    return out


def poisson(st: Stream, n: int, lam: float) -> np.ndarray:
    """Inverse-CDF Poisson draws."""
    u = st.uniform(n)
    k = np.zeros(n, dtype=np.int64)
    p = np.exp(-lam) * np.ones(n)
    c = p.copy()
    for j in range(1, 64):
        more = u > c
        if not more.any():
            break
        k += more
        p = p * lam / j
        c = c + p
    return k


def occurrences(st: Stream, n: int) -> np.ndarray:
    """min(1 + Geometric(p=0.9) failures, 255)."""
    u = st.uniform(n)
    fails = np.floor(np.log1p(-u) / np.log(0.1)).astype(np.int64)
    return np.minimum(1 + fails, 255).astype(np.uint32)


def dedup_first(sigs: np.ndarray) -> np.ndarray:
    _, first = np.unique(sigs, return_index=True)
    return sigs[np.sort(first)]


def make_case(seed: int, n_sites: int, n_queries: int, repeat_frac: float = 0.05,
              n_seeds: int = 50, lam: float = 2.0, copied_frac: float = 0.5,
              planted_into_sites: bool = True, repeat_query_frac: float = 0.0):
    """Returns (sigs uint64[n], occ uint32[n], queries uint64[q])."""
    st = Stream(seed, 1)
    n_copied = int(round(n_queries * copied_frac))
    n_rep_q = int(round(n_queries * repeat_query_frac))
    n_rand = n_queries - n_copied - n_rep_q
    n_rep_sites = int(round(n_sites * repeat_frac))
    seeds = random_sigs(st, max(n_seeds, 1))
    rep_src = seeds[st.below(n_rep_sites, len(seeds))]
    rep = substitute(st, rep_src, poisson(st, n_rep_sites, lam))
    iid = random_sigs(st, n_sites + n_sites // 16 + 64)
    pool = dedup_first(np.concatenate([rep, iid]))
    base_sites = pool[: n_sites - (n_copied if planted_into_sites else 0)]
    pick = st.below(n_copied, len(base_sites))
    copied = base_sites[pick]
    planted = substitute(st, copied, st.below(n_copied, 5))
    if planted_into_sites:
        # queries are exact copies; the planted mutants join the site set
        queries_copied = copied
        sites = dedup_first(np.concatenate([planted, base_sites]))
        extra = dedup_first(np.concatenate([sites, iid[::-1]]))
        sites = extra[:n_sites]
    else:
        queries_copied = planted
        sites = base_sites
    rep_q = substitute(st, seeds[st.below(n_rep_q, len(seeds))], st.below(n_rep_q, 3)) if n_rep_q else np.zeros(0, U64)
    rand_q = random_sigs(st, n_rand)
    queries = np.concatenate([queries_copied, rep_q, rand_q]).astype(U64)
    order = np.argsort(Stream(seed, 2).u64(len(queries)), kind="stable")
    occ = occurrences(Stream(seed, 3), len(sites))
    return sites.astype(U64), occ, queries[order]


def reference_order(sigs: np.ndarray) -> np.ndarray:
    """Sites in the order the reference's ISSLCreateIndex numbers them: ascending by their text
    (it reads a sorted site list, ISSLCreateIndex.cpp:393-417). With A<C<G<T = 0<1<2<3 and the
    first base most significant, numeric order of the reversed 2-bit groups is that order."""
    s = np.ascontiguousarray(sigs, dtype=U64)
    key = np.zeros(len(s), dtype=U64)
    for j in range(20):
        key |= ((s >> U64(2 * j)) & U64(3)) << U64(2 * (19 - j))
    return s[np.argsort(key, kind="stable")]


def sig_to_seq(sig: int, n: int = 20) -> str:
    return "".join("ACGT"[(int(sig) >> (2 * j)) & 3] for j in range(n))


def seq_to_sig(seq: str) -> int:
    v = 0
    for j, c in enumerate(seq[:20]):
        v |= {"C": 1, "G": 2, "T": 3}.get(c, 0) << (2 * j)
    return v


def masks_from_strings(lines) -> np.ndarray:
    """Slice config lines ('0/1' per position) -> position bitmasks (bit j = position j)."""
    out = []
    for line in lines:
        m = 0
        for j, c in enumerate(line.strip()):
            if c == "1":
                m |= 1 << j
        out.append(m)
    return np.array(out, dtype=U64)
