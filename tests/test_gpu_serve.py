"""Served form: requests submitted concurrently from several threads, with mixed methods,
thresholds and mismatch bounds, are batched together on the GPU; each request's result must be
the same as scoring it alone (bit for bit) and as the reference (oracle, 1e-12 relative).
Needs a GPU."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from conftest import load_case

pytestmark = pytest.mark.gpu

RTOL = 1e-12
METHODS = {"mit": 0, "cfd": 1, "mitAndCfd": 2, "mitOrCfd": 3, "avgMitCfd": 4}


@pytest.fixture(scope="module")
def c2(native, oracle):
    z, _ = load_case("c2_small")
    oix = oracle.Index.build(z["sites"], z["occ"], z["masks"])
    ix = native.Index.from_arrays(*oix.arrays())
    yield z, oix, ix
    ix.close()


def requests(q, seed, k):
    rng = np.random.default_rng(seed)
    out = []
    meths = list(METHODS)
    for _ in range(k):
        n = int(np.exp(rng.uniform(0, np.log(600))))
        pick = rng.integers(0, len(q), n)  # guides drawn with repetition from the case's queries
        out.append((q[pick].copy(), meths[rng.integers(5)], float(rng.choice([50.0, 75.0, 90.0])),
                    int(rng.choice([4, 4, 3]))))
    return out


def test_mixed_requests_equal_alone_and_oracle(native, oracle, c2):
    z, oix, ix = c2
    q = z["queries"]
    reqs = requests(q, 21, 96)
    replies = [None] * len(reqs)
    with native.Server(ix, n_slots=3, max_batch_guides=4096) as srv:
        def client(j0):
            for j in range(j0, len(reqs), 6):
                sigs, meth, thr, md = reqs[j]
                t = srv.submit(sigs, meth, thr, md)
                replies[j] = srv.wait(t)
        th = [threading.Thread(target=client, args=(i,)) for i in range(6)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        st = srv.stats()
    assert st.requests == len(reqs) and st.batches <= len(reqs)
    assert 0 < st.p50_ms <= st.p99_ms <= st.max_ms
    assert 1 <= st.peak_in_flight <= 3 and st.slots == 3
    mixed = 0
    for (sigs, meth, thr, md), rep in zip(reqs, replies):
        alone = ix.score(sigs, meth, thr, max_dist=md, distinct=False)
        r = rep.result
        assert r.code == alone.code
        np.testing.assert_array_equal(r.mit, alone.mit)
        np.testing.assert_array_equal(r.cfd, alone.cfd)
        np.testing.assert_array_equal(r.count, alone.count)
        tm, tc, cnt, _ = oix.score(sigs, METHODS[meth], thr, max_dist=md)
        ms, cs, codes = oracle.finalise(METHODS[meth], thr, tm, tc)
        assert r.code == bytes(codes)
        np.testing.assert_allclose(r.mit, ms, rtol=RTOL, atol=0)
        np.testing.assert_allclose(r.cfd, cs, rtol=RTOL, atol=0)
        np.testing.assert_array_equal(r.count, cnt)
        assert rep.info.latency_ms >= rep.info.service_ms >= 0 and rep.info.batch_guides >= len(sigs)
        mixed += rep.info.batch_requests > 1
    assert mixed > 0  # some requests were scored in a batch with others


def test_server_limits(native, c2):
    z, _, ix = c2
    q = np.resize(z["queries"], 1001)  # the case's guides, repeated
    with native.Server(ix, n_slots=2, max_batch_guides=1000) as srv:
        # above the batch limit: scored in parts, each guide's result as if scored alone
        t = srv.submit(q[:1001], "and", 75.0)
        rep = srv.wait(t)
        alone = ix.score(q[:1001], "and", 75.0, distinct=False)
        assert rep.result.code == alone.code
        assert np.array_equal(rep.result.mit, alone.mit) and np.array_equal(rep.result.cfd, alone.cfd)
        assert np.array_equal(rep.result.count, alone.count)
        assert rep.info.batch_guides <= 1000
        with pytest.raises(native.IsslError):
            srv.submit(q[:10], 9, 75.0)         # no such method
        t = srv.submit(q[:0], "and", 75.0)
        assert srv.wait(t).result.code == b""
        t = srv.submit(q[:500], "cfd", 50.0, 2)
        rep = srv.wait(t)
        alone = ix.score(q[:500], "cfd", 50.0, max_dist=2, distinct=False)
        assert rep.result.code == alone.code
    with pytest.raises(native.IsslError) as e:
        native.Server(ix, headroom_bytes=1 << 50)  # no device memory left for a slot
    assert e.value.code == -4
