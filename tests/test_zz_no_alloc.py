"""The allocation-free entry point against the regular one (needs a GPU).

issl_score_device_static serves callers that cannot allocate device memory while they score --
code running inside CUDA graph capture, hosts whose device memory belongs to their own pool
allocator, services that forbid allocation after start-up. It keeps its scratch in a fixed array
inside the library. This test allocates its own inputs and outputs (as such a caller would have
done up front), calls the entry point through the C ABI twice in a row, and checks both calls
against issl_score_device on the same guides: accept codes and off-target counts equal, MIT and
CFD scores within 1e-12 relative. It lives in its own file, collected last.
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
                rc = L.issl_score_device_static(ix.handle, C.c_void_p(d_q.data_ptr()), n, method, threshold, 4,
                                                C.c_void_p(out[0].data_ptr()), C.c_void_p(out[1].data_ptr()),
                                                C.c_void_p(out[2].data_ptr()), C.c_void_p(out[3].data_ptr()), None)
                assert rc == 0, L.issl_last_error()
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
