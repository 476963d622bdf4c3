"""Thresholds that sit on the reference's own running sums (test infrastructure).

The reference adds each guide's MIT and CFD terms one at a time in double precision, in slice
order then list order, and tests its early exit after every addition against
maximum_sum = (10000 - 100 t) / t (lib/ISSLScoringModule.cpp:225, :294-395); the accept rule
then compares 10000 / (100 + sum) with t (:404-459). For a threshold whose maximum_sum lies
within a few ulps of one of those running sums, the decision, the stopping point and so the
scores and off-target counts depend on how each addition was rounded. This module picks such
thresholds from the reference's own terms (the oracle's trace of one guide, pinned to the
reference elsewhere) so that the fixtures can be produced by the reference's binaries.

Nothing here is part of the library. make_golden.py uses it to write case_knife.npz.
"""
from __future__ import annotations

import math
from fractions import Fraction

# method names of the reference's config (util.hpp:20) and their numbers
METHODS = {"mit": 0, "cfd": 1, "mitAndCfd": 2, "mitOrCfd": 3, "avgMitCfd": 4}


def max_sum(t: float) -> float:
    """maximum_sum of ISSLScoringModule.cpp:225 in double precision."""
    return (10000.0 - t * 100) / t


def test_quantity(method: str, m: float, c: float) -> float:
    """The early-exit test of :366-395 fires iff this quantity exceeds maximum_sum."""
    if method == "mit":
        return m
    if method == "cfd":
        return c
    if method == "mitAndCfd":
        return min(m, c)
    if method == "mitOrCfd":
        return max(m, c)
    return (m + c) / 2.0


def running(terms) -> list:
    """Running sums rounded after every addition, as the reference accumulates them."""
    out, s = [], 0.0
    for x in terms:
        s += float(x)
        out.append(s)
    return out


def exact_running(terms) -> list:
    """Running sums without rounding, each rounded once to a double at the end."""
    out, s = [], Fraction(0)
    for x in terms:
        s += Fraction(float(x))
        out.append(float(s))
    return out


def thresholds_near(x: float, ulps: int = 3, steps: int = 40) -> list:
    """Thresholds t in (0, 100] whose maximum_sum is within `ulps` ulps of x (nearest first)."""
    if not (x > 0 and math.isfinite(x)):
        return []
    t0 = 10000.0 / (x + 100.0)
    lo, hi = x - ulps * math.ulp(x), x + ulps * math.ulp(x)
    found = {}
    for direction in (-math.inf, math.inf):
        t = t0
        for _ in range(steps):
            m = max_sum(t)
            if lo <= m <= hi and 0 < t <= 100:
                found[t] = abs(m - x)
            t = math.nextafter(t, direction)
    return [t for t, _ in sorted(found.items(), key=lambda kv: (kv[1], kv[0]))]


def pick_points(method: str, mit_terms, cfd_terms):
    """Positions k (0-based hit index) worth aiming a threshold at: the last hit (the accept rule
    on the full sums, no exit), and an interior hit -- the first one past a quarter of the hits
    where the rounded and exact running quantities differ, else the middle one.
    Returns (k, rounded quantity, exact quantity) triples."""
    rm, rc = running(mit_terms), running(cfd_terms)
    em, ec = exact_running(mit_terms), exact_running(cfd_terms)
    n = len(rm)
    qr = [test_quantity(method, a, b) for a, b in zip(rm, rc)]
    qe = [test_quantity(method, a, b) for a, b in zip(em, ec)]
    points = [n - 1]
    inner = next((k for k in range(n // 4, n - 1) if qr[k] != qe[k]), n // 2)
    if inner != n - 1:
        points.append(inner)
    return [(k, qr[k], qe[k]) for k in points]


def entries(trace, guide_ids, per_point: int = 4):
    """Knife-edge (guide, method, threshold) triples. trace(g) gives the guide's (mit_terms,
    cfd_terms, occurrences). Per guide, method and aimed hit: the thresholds whose maximum_sum
    is nearest the reference's rounded quantity there, plus every threshold whose maximum_sum
    falls between the rounded and the exact quantity (where a decision taken on exact sums
    would differ from the reference's)."""
    out = []
    for g in guide_ids:
        mt, ct, _ = trace(g)
        if len(mt) == 0:
            continue
        for method in METHODS:
            seen = set()
            for k, q_round, q_exact in pick_points(method, mt, ct):
                chosen = thresholds_near(q_round)[:per_point]
                if q_round != q_exact:
                    a, b = sorted((q_round, q_exact))
                    chosen += [t for t in thresholds_near(q_exact, ulps=8) if a <= max_sum(t) <= b]
                for t in chosen:
                    if t not in seen:
                        seen.add(t)
                        out.append((int(g), method, float(t), int(k)))
    return out


def exact_decision_differs(method: str, t: float, mit_terms, cfd_terms) -> bool:
    """Would a scorer that tests and decides on exactly summed (then rounded) totals reach a
    different stopping point or accept code than the reference's rounded running sums?"""
    def outcome(rm, rc):
        M = max_sum(t)
        stop = len(rm) - 1
        for k in range(len(rm)):
            if test_quantity(method, rm[k], rc[k]) > M:
                stop = k
                break
        m = 10000.0 / (100.0 + rm[stop])
        c = 10000.0 / (100.0 + rc[stop])
        rej = {"mit": m < t, "cfd": c < t, "mitAndCfd": m < t and c < t, "mitOrCfd": m < t or c < t,
               "avgMitCfd": (m + c) / 2 < t}[method]
        return stop, rej

    return outcome(running(mit_terms), running(cfd_terms)) != outcome(exact_running(mit_terms),
                                                                      exact_running(cfd_terms))
