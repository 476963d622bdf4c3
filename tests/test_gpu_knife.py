"""Thresholds on the reference's own running sums (needs a GPU).

The reference adds a guide's terms one at a time in double precision and stops at the first
addition whose running sum passes maximum_sum (lib/ISSLScoringModule.cpp:225, :366-395); the
library sums the same terms exactly. case_knife.npz holds (guide, method, threshold) entries whose
maximum_sum lies within a few ulps of one of the guide's running sums -- about a third of them
placed where a decision taken on exact sums would differ from the reference's -- each scored by
the reference's ISSLScoringModule (scores, accept code) and ISSLScoreOfftargets (off-target count).

Bar: accept codes and counts equal to the reference's for every entry, scores within 1e-12
relative; every entry where exact sums would decide differently is rescored one addition at a
time (issl_score_stats.replayed), in every slice-wave split.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_case

pytestmark = pytest.mark.gpu

RTOL = 1e-12
NAMES = ["mit", "cfd", "mitAndCfd", "mitOrCfd", "avgMitCfd"]


@pytest.fixture(scope="module")
def knife(oracle):
    z, meta = load_case("knife")
    arrays = oracle.Index.build(z["sites"], z["occ"], z["masks"]).arrays()
    return z, meta, arrays


def _check(tag, i, z, mit, cfd, code, count):
    g, m, t = int(z["guide"][i]), NAMES[int(z["method"][i])], float(z["threshold"][i])
    where = f"{tag}: entry {i} (guide {g}, {m}, t={t!r})"
    assert code == int(z["code"][i]), where + ": accept code"
    assert count == int(z["count"][i]), where + ": off-target count"
    np.testing.assert_allclose(mit, z["mit"][i], rtol=RTOL, atol=0, err_msg=where)
    np.testing.assert_allclose(cfd, z["cfd"][i], rtol=RTOL, atol=0, err_msg=where)


@pytest.mark.parametrize("first_wave", [1, 0, 2])
def test_knife_edge_plain(native, knife, first_wave):
    z, meta, arrays = knife
    q = z["queries"]
    with native.Index.from_arrays(*arrays) as ix:
        ix.set_tuning(first_wave=first_wave)
        replayed_where_needed = 0
        for i in range(len(z["guide"])):
            g = int(z["guide"][i])
            res = ix.score(q[g:g + 1], NAMES[int(z["method"][i])], float(z["threshold"][i]))
            _check(f"plain first_wave={first_wave}", i, z, res.mit[0], res.cfd[0], res.code[0], int(res.count[0]))
            if z["exact_differs"][i]:
                assert ix.last_stats().replayed == 1, f"entry {i}: exact sums decide differently, not rescored"
                replayed_where_needed += 1
        assert replayed_where_needed == int(z["exact_differs"].sum()) > 100


def test_knife_edge_batched(native, knife):
    """All entries as one-guide sets of one batch, each with its own method and threshold."""
    z, meta, arrays = knife
    sigs = z["queries"][z["guide"]]
    sets = [(1, NAMES[int(m)], float(t), 4) for m, t in zip(z["method"], z["threshold"])]
    with native.Index.from_arrays(*arrays) as ix:
        with native.Batch(ix) as bt:
            for _ in range(2):  # the second call replays the captured graph
                res = bt.score(sigs, sets)
                for i in range(len(sets)):
                    _check("batched", i, z, res.mit[i], res.cfd[i], res.code[i], int(res.count[i]))
                assert bt.stats().replayed >= int(z["exact_differs"].sum())
