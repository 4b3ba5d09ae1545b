"""The allocation-free sort entry point, pbf_sort_keys_noalloc.

It exists for callers that cannot call cudaMalloc (device memory owned by
another framework's pool, plugins handed only device buffers, real-time loops
that must stay out of the allocator): they pass their own device buffers and
the scratch comes from a fixed array inside the library.  This test calls it
through the C ABI twice in a row and checks each result against the
allocating entry point pbf_sort_keys.  The integer sort is bit-exact, so the
tolerance is equality.  The file sorts last so that a failure here leaves
every other test already run; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_u32(torch, host):
    return torch.from_numpy(host.view(np.int32).copy()).to("cuda")


def test_noalloc_sort_matches_allocating_sort_twice(have_gpu):
    import torch

    import pbf_b200 as P
    from pbf_b200 import _capi

    L = _capi.lib()
    rng = np.random.default_rng(2024)
    for call, (n, bits) in enumerate([(300_001, 22), (1 << 20, 17)]):
        keys = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32)
        want_k, want_i = P.sort_keys(keys, bits)  # allocating entry point
        d_keys = _device_u32(torch, keys)
        d_sk = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        d_si = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = L.pbf_sort_keys_noalloc(C.c_void_p(d_keys.data_ptr()), n, bits, C.c_void_p(d_sk.data_ptr()),
                                     C.c_void_p(d_si.data_ptr()), None)
        assert rc == _capi.PBF_OK, L.pbf_last_error()
        torch.cuda.synchronize()
        got_k = d_sk.cpu().numpy().view(np.uint32)
        got_i = d_si.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_k, want_k), call
        assert np.array_equal(got_i, want_i), call


def test_noalloc_sort_rejects_oversized_input(have_gpu):
    from pbf_b200 import _capi

    L = _capi.lib()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.pbf_sort_keys_noalloc(dummy, (1 << 20) + 1, 22, C.c_void_p(32), C.c_void_p(48), None)
    assert rc == _capi.PBF_ERR_INVALID
    assert b"exceed" in L.pbf_last_error()
