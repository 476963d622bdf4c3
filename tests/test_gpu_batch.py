"""Batched form and scan tuning: many guide sets with their own method / threshold / mismatch
bound in one graph-captured pass must give every guide the result of a call of its own (bit for
bit, since the sums are exact) and the reference's result (oracle, 1e-12 relative). Needs a GPU."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_case

pytestmark = pytest.mark.gpu

RTOL = 1e-12
METHODS = {"mit": 0, "cfd": 1, "mitAndCfd": 2, "mitOrCfd": 3, "avgMitCfd": 4}


@pytest.fixture(scope="module")
def c2(native, oracle):
    """The slice-10-37 small case (the batched form's slice configuration)."""
    z, _ = load_case("c2_small")
    oix = oracle.Index.build(z["sites"], z["occ"], z["masks"])
    ix = native.Index.from_arrays(*oix.arrays())
    yield z, oix, ix
    ix.close()


def uneven_sets(q, seed):
    """Log-uniform set sizes over the queries, methods / thresholds / bounds drawn per set."""
    rng = np.random.default_rng(seed)
    sizes, left = [], len(q)
    while left > 0:
        s = min(left, int(np.exp(rng.uniform(np.log(1), np.log(400)))))
        sizes.append(s)
        left -= s
    meths = list(METHODS)
    return [(s, meths[rng.integers(5)], float(rng.choice([50.0, 75.0, 90.0, 99.0])), int(rng.choice([4, 4, 3, 2])))
            for s in sizes]


def check_batch_against_singles(ix, oracle, oix, q, sets, res):
    b = 0
    for count, meth, thr, md in sets:
        sl = slice(b, b + count)
        single = ix.score(q[sl], meth, thr, max_dist=md, distinct=False)
        assert res.code[sl] == single.code, (meth, thr, md)
        np.testing.assert_array_equal(res.mit[sl], single.mit)
        np.testing.assert_array_equal(res.cfd[sl], single.cfd)
        np.testing.assert_array_equal(res.count[sl], single.count)
        tm, tc, cnt, _ = oix.score(q[sl], METHODS[meth], thr, max_dist=md)
        ms, cs, codes = oracle.finalise(METHODS[meth], thr, tm, tc)
        assert res.code[sl] == bytes(codes)
        np.testing.assert_allclose(res.mit[sl], ms, rtol=RTOL, atol=0)
        np.testing.assert_allclose(res.cfd[sl], cs, rtol=RTOL, atol=0)
        np.testing.assert_array_equal(res.count[sl], cnt)
        b += count


def test_batch_of_uneven_sets_equals_single_calls_and_oracle(native, oracle, c2):
    z, oix, ix = c2
    q = z["queries"]
    sets = uneven_sets(q, 11)
    assert len(sets) > 5
    with native.Batch(ix) as bt:
        res = bt.score(q, sets)
        check_batch_against_singles(ix, oracle, oix, q, sets, res)
        st = bt.stats()
        assert st.launches >= 18 and st.total_ms > 0


def test_graph_replays_for_new_batches_and_regrows(native, oracle, c2):
    z, oix, ix = c2
    q = z["queries"]
    with native.Batch(ix) as bt:
        small = q[:300]
        s1 = uneven_sets(small, 1)
        r1 = bt.score(small, s1)
        rev = small[::-1].copy()
        s2 = uneven_sets(rev, 2)
        r2 = bt.score(rev, s2)  # same capacities: the captured graph is replayed
        check_batch_against_singles(ix, oracle, oix, small, s1, r1)
        check_batch_against_singles(ix, oracle, oix, rev, s2, r2)
        big = np.concatenate([q, q[:2000]])  # larger than the first capacity: re-captured
        s3 = uneven_sets(big, 3)
        r3 = bt.score(big, s3)
        check_batch_against_singles(ix, oracle, oix, big, s3, r3)
        r1b = bt.score(small, s1)
        assert r1b.code == r1.code
        np.testing.assert_array_equal(r1b.mit, r1.mit)
        np.testing.assert_array_equal(r1b.cfd, r1.cfd)


def test_batch_device_buffers(native, c2):
    import torch
    z, _, ix = c2
    q = z["queries"][:500]
    sets = uneven_sets(q, 5)
    n = len(q)
    d_q = torch.from_numpy(q.view(np.int64)).cuda()
    d_mit = torch.empty(n, dtype=torch.float64, device="cuda")
    d_cfd = torch.empty(n, dtype=torch.float64, device="cuda")
    d_code = torch.empty(n, dtype=torch.uint8, device="cuda")
    d_cnt = torch.empty(n, dtype=torch.int64, device="cuda")
    with native.Batch(ix) as bt:
        bt.score_device(d_q.data_ptr(), n, sets, d_mit.data_ptr(), d_cfd.data_ptr(), d_code.data_ptr(),
                        d_cnt.data_ptr())
        host = bt.score(q, sets)
    assert bytes(d_code.cpu().numpy()) == host.code
    np.testing.assert_array_equal(d_mit.cpu().numpy(), host.mit)
    np.testing.assert_array_equal(d_cfd.cpu().numpy(), host.cfd)
    np.testing.assert_array_equal(d_cnt.cpu().numpy().view(np.uint64), host.count)


def test_batch_with_empty_sets_and_bad_tables(native, c2):
    z, _, ix = c2
    q = z["queries"][:50]
    with native.Batch(ix) as bt:
        r = bt.score(q, [(0, "mit", 75.0, 4), (50, "and", 75.0, 4), (0, "cfd", 50.0, 2)])
        single = ix.score(q, "and", 75.0, distinct=False)
        assert r.code == single.code
        np.testing.assert_array_equal(r.mit, single.mit)
        with pytest.raises(native.IsslError):
            bt.score(q, [(49, "and", 75.0, 4)])  # counts do not add up
        with pytest.raises(native.IsslError):
            bt.score(q, [(50, "and", 75.0, 5)])  # max_dist beyond 4
        with pytest.raises(native.IsslError):
            bt.score(q, [(50, 9, 75.0, 4)])      # no such method


@pytest.mark.parametrize("tuning", [((256, 256, 256), 2, 0, 0), ((512, 1024, 256), 4, 0, 3), ((1024, 512, 512), 3, 2, 1),
                                    ((1024, 1024, 1024), 2, 1, 36), ((1024, 1024, 1024), 3, 0, 37)])
def test_results_do_not_depend_on_tuning(native, c2, tuning):
    z, _, ix = c2
    q = z["queries"]
    base = ix.score(q, "and", 90.0)
    chunk, stages, bps, fw = tuning
    ix.set_tuning(chunk, stages, bps, fw)
    try:
        assert ix.get_tuning().as_tuple() == (tuple(chunk), stages, bps, fw)
        r = ix.score(q, "and", 90.0)
        with native.Batch(ix) as bt:
            rb = bt.score(q, [(len(q), "and", 90.0, 4)])
    finally:
        ix.set_tuning()
    for x in (r, rb):
        assert x.code == base.code
        np.testing.assert_array_equal(x.mit, base.mit)
        np.testing.assert_array_equal(x.cfd, base.cfd)
        np.testing.assert_array_equal(x.count, base.count)
    assert r.distinct == base.distinct


def test_guide_chunks_give_the_same_results(native, c2, monkeypatch):
    z, _, ix = c2
    q = z["queries"]
    whole = ix.score(q, "and", 90.0)
    sets = uneven_sets(q, 7)
    with native.Batch(ix) as bt:
        whole_b = bt.score(q, sets)
    monkeypatch.setenv("ISSL_MAX_GUIDES_PER_RUN", "37")
    parts = ix.score(q, "and", 90.0)
    with native.Batch(ix) as bt:
        parts_b = bt.score(q, sets)
    for a, b in [(whole, parts), (whole_b, parts_b)]:
        assert a.code == b.code and a.distinct == b.distinct
        np.testing.assert_array_equal(a.mit, b.mit)
        np.testing.assert_array_equal(a.cfd, b.cfd)
        np.testing.assert_array_equal(a.count, b.count)


def test_trim_then_score_again(native, c2):
    z, _, ix = c2
    q = z["queries"]
    a = ix.score(q, "or", 75.0)
    ix.trim()
    b = ix.score(q, "or", 75.0)
    assert a.code == b.code and a.distinct == b.distinct
    np.testing.assert_array_equal(a.mit, b.mit)
    np.testing.assert_array_equal(a.cfd, b.cfd)


def test_invalid_tuning_rejected(native, c2):
    _, _, ix = c2
    for bad in [((300, 1024, 1024), 3, 0, 1), ((1024, 1024, 1024), 5, 0, 1), ((1024, 1024, 1024), 1, 0, 1),
                ((1024, 1024, 1024), 3, 0, 65)]:
        with pytest.raises(native.IsslError):
            ix.set_tuning(*bad)
    assert ix.get_tuning().as_tuple() == ((1024, 1024, 1024), 2, 0, 1)  # the default is kept


def test_autotune_and_cache(native, c2, tmp_path):
    import torch
    z, _, ix = c2
    d = torch.from_numpy(z["queries"].view(np.int64)).cuda()
    cache = str(tmp_path / "tune.txt")
    try:
        t, rep = ix.autotune(d.data_ptr(), len(d), "and", 75.0, 4, cache)
        assert rep.from_cache == 0 and rep.configs_timed >= 6
        assert 0 < rep.best_ms <= rep.default_ms * 1.0001
        assert sum(rep.class_probes) > 0
        assert ix.get_tuning().as_tuple() == t.as_tuple()
        ix.set_tuning()
        t2, rep2 = ix.autotune(d.data_ptr(), len(d), "and", 75.0, 4, cache)
        assert rep2.from_cache == 1 and t2.as_tuple() == t.as_tuple()
    finally:
        ix.set_tuning()
