"""Host-list index (issl_open_mapped, the role of the reference's memory-mapped module
lib/ISSLScoringModuleMMF.cpp:73-128): the list entries and bit-sliced codes stay in page-locked
host memory and every call streams them to the device in windows of slices. Results must equal
the resident index's bit for bit (the sums are exact, so the wave split cannot change them) and
the oracle's within 1e-12. Needs a GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import load_case

pytestmark = pytest.mark.gpu

RTOL = 1e-12
METHODS = {"mit": 0, "cfd": 1, "mitAndCfd": 2, "mitOrCfd": 3, "avgMitCfd": 4}
ISSL_ERR_UNSUPPORTED = -7


@pytest.fixture(scope="module")
def c1(native, oracle, tmp_path_factory):
    """The slice-8-20 small case, resident and as a file."""
    z, _ = load_case("c1_small")
    oix = oracle.Index.build(z["sites"], z["occ"], z["masks"])
    ix = native.Index.from_arrays(*oix.arrays())
    path = str(tmp_path_factory.mktemp("mapped") / "c1.issl")
    ix.save(path)
    yield z, oix, ix, path
    ix.close()


def assert_same(a, b):
    assert a.code == b.code
    np.testing.assert_array_equal(a.mit, b.mit)
    np.testing.assert_array_equal(a.cfd, b.cfd)
    np.testing.assert_array_equal(a.count, b.count)
    assert a.distinct == b.distinct


@pytest.mark.parametrize("window", [1, 3, 7, 20])
def test_mapped_equals_resident_and_oracle(native, oracle, c1, window):
    z, oix, ix, path = c1
    mx = native.Index.open_mapped(path, window_slices=window)
    try:
        inf = mx.info()
        assert inf.window_slices == window
        assert inf.host_bytes > 0
        assert inf.device_bytes < ix.info().device_bytes
        q = z["queries"]
        for meth, thr, md in [("mitAndCfd", 75.0, 4), ("mitOrCfd", 50.0, 4), ("mit", 90.0, 3),
                              ("cfd", 75.0, 4), ("avgMitCfd", 99.0, 2)]:
            assert_same(mx.score(q, meth, thr, max_dist=md), ix.score(q, meth, thr, max_dist=md))
        res = mx.score(q, "mitAndCfd", 75.0)
        tm, tc, cnt, _ = oix.score(q, 2, 75.0)
        ms, cs, codes = oracle.finalise(2, 75.0, tm, tc)
        assert res.code == bytes(codes)
        np.testing.assert_allclose(res.mit, ms, rtol=RTOL, atol=0)
        np.testing.assert_allclose(res.cfd, cs, rtol=RTOL, atol=0)
        np.testing.assert_array_equal(res.count, cnt)
    finally:
        mx.close()


def test_mapped_with_first_wave_and_repeated_calls(native, c1):
    """Windows cut inside both slice waves; several calls in a row reuse the two windows."""
    z, _, ix, path = c1
    mx = native.Index.open_mapped(path, window_slices=3)
    try:
        mx.set_tuning(first_wave=4)
        ix.set_tuning(first_wave=4)
        q = z["queries"]
        ref = ix.score(q, "mitAndCfd", 75.0)
        for _ in range(3):
            assert_same(mx.score(q, "mitAndCfd", 75.0), ref)
        part = q[: len(q) // 3]
        assert_same(mx.score(part, "cfd", 50.0), ix.score(part, "cfd", 50.0))
    finally:
        ix.set_tuning(first_wave=1)
        mx.close()


def test_mapped_export_equals_resident(native, c1):
    _, _, ix, path = c1
    mx = native.Index.open_mapped(path, window_slices=2)
    try:
        for a, b in zip(mx.export(), ix.export()):
            np.testing.assert_array_equal(a, b)
    finally:
        mx.close()


def test_mapped_batch_form_equals_singles(native, c1):
    """The batch form captures the window copies (a second stream) into its graph."""
    z, _, ix, path = c1
    mx = native.Index.open_mapped(path, window_slices=4)
    try:
        q = z["queries"]
        n = len(q)
        sets = [(n // 4, "mitAndCfd", 75.0, 4), (n // 4, "cfd", 90.0, 3), (n - 2 * (n // 4), "mit", 50.0, 4)]
        with native.Batch(mx) as b:
            for _ in range(2):  # the second call replays the captured graph
                res = b.score(q, sets)
                s0 = 0
                for count, meth, thr, md in sets:
                    single = ix.score(q[s0:s0 + count], meth, thr, max_dist=md, distinct=False)
                    assert res.code[s0:s0 + count] == single.code
                    np.testing.assert_array_equal(res.mit[s0:s0 + count], single.mit)
                    np.testing.assert_array_equal(res.cfd[s0:s0 + count], single.cfd)
                    np.testing.assert_array_equal(res.count[s0:s0 + count], single.count)
                    s0 += count
    finally:
        mx.close()


def test_mapped_synthetic_index_with_repeats(native, tmp_path):
    """A 3M-site index with repeat families (heavy buckets, guides with many hits): windows of
    several megabytes per slice, guide chunks and slice waves all on the streamed path."""
    spec = native.SynthSpec(seed=77, n_sites=3_000_000, slice_config="slice-8-20", n_queries=20_000,
                            repeat_query_frac=0.2)
    ix, q = native.Index.synth(spec)
    try:
        path = str(tmp_path / "synth.issl")
        ix.save(path)
        mx = native.Index.open_mapped(path, window_slices=6)
        try:
            assert_same(mx.score(q, "mitAndCfd", 75.0), ix.score(q, "mitAndCfd", 75.0))
            assert_same(mx.score(q, "mitOrCfd", 90.0, max_dist=3), ix.score(q, "mitOrCfd", 90.0, max_dist=3))
        finally:
            mx.close()
    finally:
        ix.close()


def test_static_entry_point_refuses_mapped_index(native, c1):
    import torch

    _, _, _, path = c1
    mx = native.Index.open_mapped(path, window_slices=2)
    try:
        L = native.lib()
        d_q = torch.zeros(4, dtype=torch.int64, device="cuda")
        d_code = torch.zeros(4, dtype=torch.uint8, device="cuda")
        rc = L.issl_score_device_static(mx.handle, C.c_void_p(d_q.data_ptr()), 4, 2, 75.0, 4, None, None,
                                        C.c_void_p(d_code.data_ptr()), None, None)
        assert rc == ISSL_ERR_UNSUPPORTED
        assert b"host memory" in L.issl_last_error()
    finally:
        mx.close()


def test_list_placement_round_trip_with_live_batch_context(native):
    """Lists moved to host memory and back on an open index: plain calls and a batch context
    created before the move (its graph is re-captured) keep giving the resident results."""
    spec = native.SynthSpec(seed=78, n_sites=1_000_000, slice_config="slice-10-37", n_queries=8_000,
                            repeat_query_frac=0.2)
    ix, q = native.Index.synth(spec)
    try:
        sets = [(3_000, "mitAndCfd", 75.0, 4), (5_000, "cfd", 90.0, 3)]
        ref = ix.score(q, "mitAndCfd", 75.0)
        with native.Batch(ix) as b:
            ref_b = b.score(q, sets)
            ix.set_list_placement(5)
            assert ix.info().window_slices == 5 and ix.info().host_bytes > 0
            assert_same(ix.score(q, "mitAndCfd", 75.0), ref)
            got_b = b.score(q, sets)
            assert got_b.code == ref_b.code
            np.testing.assert_array_equal(got_b.mit, ref_b.mit)
            np.testing.assert_array_equal(got_b.cfd, ref_b.cfd)
            np.testing.assert_array_equal(got_b.count, ref_b.count)
            ix.set_list_placement(0)
            assert ix.info().window_slices == 0 and ix.info().host_bytes == 0
            assert_same(ix.score(q, "mitAndCfd", 75.0), ref)
            got_b = b.score(q, sets)
            assert got_b.code == ref_b.code
            np.testing.assert_array_equal(got_b.mit, ref_b.mit)
    finally:
        ix.close()
