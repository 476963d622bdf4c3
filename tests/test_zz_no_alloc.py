"""The allocation-free entry point against the regular one (needs a GPU).

issl_score_device_static serves callers that cannot allocate device memory while they score --
hosts whose device memory belongs to their own pool allocator (a framework's caching allocator, a
fixed arena on a shared GPU), services that forbid allocation after start-up. It keeps its
scratch in a fixed array inside the library. These tests allocate their own inputs and outputs
(as such a caller would have done up front) and call the entry point through the C ABI:
  * twice in a row, against issl_score_device on the same guides: accept codes and off-target
    counts equal, MIT and CFD scores within 1e-12 relative; the device's free memory does not
    change across a call;
  * on the knife-edge fixture, against the reference itself: the entry point adds each guide's
    terms one at a time in the reference's order, so scores, codes and counts equal the
    reference's bit for bit;
  * with a guide beyond the per-guide hit limit: the call reports ISSL_ERR_UNSUPPORTED and every
    other guide's results are still those of issl_score_device.
They live in a file of their own, collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _device_outputs(torch, n, dev):
    return (torch.empty(n, dtype=torch.float64, device=dev), torch.empty(n, dtype=torch.float64, device=dev),
            torch.empty(n, dtype=torch.uint8, device=dev), torch.empty(n, dtype=torch.int64, device=dev))


def test_static_entry_point_matches_regular(native):
    import torch
    dev = torch.device("cuda", 0)
    L = native.lib()
    spec = native.SynthSpec(seed=29, n_sites=300_000, slice_config="slice-8-20", n_queries=700,
                            n_repeat_seeds=100, repeat_query_frac=0.1)
    ix, q = native.Index.synth(spec, device=0)
    with ix:
        n = len(q)
        d_q = torch.from_numpy(q.view(np.int64)).to(dev)
        ref = _device_outputs(torch, n, dev)
        for method, threshold in [(2, 75.0), (4, 90.0), (1, 99.0)]:
            ix.score_device(d_q.data_ptr(), n, method, threshold, 4, ref[0].data_ptr(), ref[1].data_ptr(),
                            ref[2].data_ptr(), ref[3].data_ptr())
            torch.cuda.synchronize()
            runs = []
            for _ in range(2):  # two calls in a row share the static scratch
                out = _device_outputs(torch, n, dev)
                torch.cuda.synchronize()
                free_before = torch.cuda.mem_get_info(dev)[0]
                rc = L.issl_score_device_static(ix.handle, C.c_void_p(d_q.data_ptr()), n, method, threshold, 4,
                                                C.c_void_p(out[0].data_ptr()), C.c_void_p(out[1].data_ptr()),
                                                C.c_void_p(out[2].data_ptr()), C.c_void_p(out[3].data_ptr()), None)
                assert rc == 0, L.issl_last_error()
                if runs:  # after the first call (which may load the library's device code)
                    assert torch.cuda.mem_get_info(dev)[0] == free_before, "the call changed free device memory"
                runs.append([t.cpu().numpy() for t in out])
            want = [t.cpu().numpy() for t in ref]
            for got in runs:
                assert np.array_equal(got[2], want[2]), "accept codes differ"
                assert np.array_equal(got[3], want[3]), "off-target counts differ"
                np.testing.assert_allclose(got[0], want[0], rtol=RTOL, atol=0)
                np.testing.assert_allclose(got[1], want[1], rtol=RTOL, atol=0)
        # more guides than the entry point takes is an argument error, before any device work
        rc = L.issl_score_device_static(ix.handle, C.c_void_p(d_q.data_ptr()), (1 << 20) + 1, 2, 75.0, 4,
                                        C.c_void_p(ref[0].data_ptr()), C.c_void_p(ref[1].data_ptr()),
                                        C.c_void_p(ref[2].data_ptr()), C.c_void_p(ref[3].data_ptr()), None)
        assert rc == -1 and b"at most" in L.issl_last_error()


def _static(L, ix, d_q, n, method, threshold, out):
    return L.issl_score_device_static(ix.handle, C.c_void_p(d_q.data_ptr()), n, method, threshold, 4,
                                      C.c_void_p(out[0].data_ptr()), C.c_void_p(out[1].data_ptr()),
                                      C.c_void_p(out[2].data_ptr()), C.c_void_p(out[3].data_ptr()), None)


def test_static_entry_point_equals_reference_on_knife_edge(native, oracle):
    """Thresholds on the reference's own running sums: bit-for-bit the reference's results."""
    import torch
    from conftest import load_case
    dev = torch.device("cuda", 0)
    L = native.lib()
    z, _ = load_case("knife")
    arrays = oracle.Index.build(z["sites"], z["occ"], z["masks"]).arrays()
    with native.Index.from_arrays(*arrays) as ix:
        d_all = torch.from_numpy(z["queries"].view(np.int64)).to(dev)
        out = _device_outputs(torch, 1, dev)
        for i in range(len(z["guide"])):
            g = int(z["guide"][i])
            rc = _static(L, ix, d_all[g:g + 1], 1, int(z["method"][i]), float(z["threshold"][i]), out)
            assert rc == 0, L.issl_last_error()
            got = [t.cpu().numpy()[0] for t in out]
            assert (got[0], got[1], int(got[2]), int(got[3])) == \
                (z["mit"][i], z["cfd"][i], int(z["code"][i]), int(z["count"][i])), f"entry {i}"


def test_static_entry_point_hit_limit(native):
    """A guide with more owned hits than the per-guide limit makes the call fail with
    ISSL_ERR_UNSUPPORTED; the other guides of the call are scored as issl_score_device scores them."""
    import torch
    import synth
    from cracklingplusplus_gpu_b200.slice_configs import slice_masks
    dev = torch.device("cuda", 0)
    L = native.lib()
    st = synth.Stream(41, 1)
    centre = int(synth.random_sigs(st, 1)[0])
    k = 1 + st.below(9000, 4)  # 1..4 substitutions: every mutant is a hit of the centre guide
    mutants = synth.substitute(st, np.full(9000, centre, np.uint64), k)
    near = synth.dedup_first(mutants[mutants != np.uint64(centre)])
    assert len(near) > 4096  # ISSL_STATIC_MAX_HITS
    background = synth.random_sigs(st, 20000)
    sites = synth.dedup_first(np.concatenate([near, background]))
    occ = np.ones(len(sites), np.uint32)
    queries = np.concatenate([np.array([centre], np.uint64), synth.random_sigs(st, 200), near[:50]])
    with native.Index.build(sites, occ, np.array(slice_masks("slice-8-20"), np.uint64)) as ix:
        n = len(queries)
        d_q = torch.from_numpy(queries.view(np.int64)).to(dev)
        ref = _device_outputs(torch, n, dev)
        ix.score_device(d_q.data_ptr(), n, 2, 75.0, 4, ref[0].data_ptr(), ref[1].data_ptr(), ref[2].data_ptr(),
                        ref[3].data_ptr())
        torch.cuda.synchronize()
        assert ix.last_stats().hits > 4096  # the regular entry point has no per-guide limit
        out = _device_outputs(torch, n, dev)
        rc = _static(L, ix, d_q, n, 2, 75.0, out)
        assert rc == -7 and b"off-target hits" in L.issl_last_error()
        want = [t.cpu().numpy()[1:] for t in ref]
        got = [t.cpu().numpy()[1:] for t in out]
        assert np.array_equal(got[2], want[2]) and np.array_equal(got[3], want[3])
        np.testing.assert_allclose(got[0], want[0], rtol=RTOL, atol=0)
        np.testing.assert_allclose(got[1], want[1], rtol=RTOL, atol=0)
