"""The allocation-free sort entry point, pbf_sort_keys_noalloc.

It exists for callers that cannot call cudaMalloc (device memory owned by
another framework's pool, plugins handed only device buffers, real-time loops
that must stay out of the allocator): they pass their own device buffers and
the scratch comes from a fixed array inside the library.  The GPU tests call
it through the C ABI twice in a row and check each result against the
allocating entry point pbf_sort_keys.  The integer sort is bit-exact, so the
tolerance is equality.  Every rejection test hands it real device buffers of
the size it names, so that a regression in an argument check gives a wrong
return code rather than a kernel running on addresses that do not exist.  The
file sorts last so that a failure here leaves every other test already run; it
also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest


def _device_u32(torch, host):
    return torch.from_numpy(host.view(np.int32).copy()).to("cuda")


def _ptr(t, offset_words=0):
    return C.c_void_p(t.data_ptr() + 4 * offset_words)


@pytest.mark.gpu
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
        rc = L.pbf_sort_keys_noalloc(_ptr(d_keys), n, bits, _ptr(d_sk), _ptr(d_si), None)
        assert rc == _capi.PBF_OK, L.pbf_last_error()
        torch.cuda.synchronize()
        got_k = d_sk.cpu().numpy().view(np.uint32)
        got_i = d_si.cpu().numpy().view(np.uint32)
        assert np.array_equal(got_k, want_k), call
        assert np.array_equal(got_i, want_i), call


@pytest.mark.gpu
def test_noalloc_sort_rejects_oversized_input(have_gpu):
    import torch

    from pbf_b200 import _capi

    L = _capi.lib()
    n = (1 << 20) + 1  # one key past the fixed scratch
    bufs = [torch.zeros(n, dtype=torch.int32, device="cuda") for _ in range(3)]
    torch.cuda.synchronize()
    rc = L.pbf_sort_keys_noalloc(_ptr(bufs[0]), n, 22, _ptr(bufs[1]), _ptr(bufs[2]), None)
    torch.cuda.synchronize()
    assert rc == _capi.PBF_ERR_INVALID
    assert b"exceed" in L.pbf_last_error()


@pytest.mark.gpu
def test_noalloc_sort_rejects_overlapping_buffers(have_gpu):
    """keys, sorted keys and sorted ids: any two that share a word are refused
    (with 9 key bits the sort makes two passes, with 8 one; an odd count writes
    the first pass into the outputs while the keys are still being read)."""
    import torch

    from pbf_b200 import _capi

    L = _capi.lib()
    n = 4096
    big = torch.zeros(4 * n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    cases = [(0, 0, 2 * n), (0, 2 * n, 0), (0, n, n), (0, n // 2, 2 * n), (0, 2 * n, 2 * n + n - 1),
             (n, n // 2, 3 * n), (2 * n, 3 * n, 2 * n + 1)]
    for bits in (8, 9):
        for k, sk, si in cases:
            rc = L.pbf_sort_keys_noalloc(_ptr(big, k), n, bits, _ptr(big, sk), _ptr(big, si), None)
            assert rc == _capi.PBF_ERR_INVALID, (bits, k, sk, si)
            assert b"overlap" in L.pbf_last_error()
    torch.cuda.synchronize()


def test_noalloc_sort_argument_checks_on_cpu():
    """The size and overlap checks come before any CUDA call, so they can be
    exercised where there is no GPU at all.  Skipped on a machine with a GPU,
    where the GPU tests above cover the same checks with device buffers."""
    import torch

    from pbf_b200 import _capi

    if torch.cuda.is_available():
        pytest.skip("covered by the device-buffer tests on a GPU")
    L = _capi.lib()
    n = 1 << 12
    host = np.zeros(4 * n, dtype=np.uint32)
    base = host.ctypes.data

    def at(w):
        return C.c_void_p(base + 4 * w)

    assert L.pbf_sort_keys_noalloc(at(0), n, 9, at(0), at(2 * n), None) == _capi.PBF_ERR_INVALID
    assert L.pbf_sort_keys_noalloc(at(0), n, 9, at(2 * n), at(0), None) == _capi.PBF_ERR_INVALID
    assert L.pbf_sort_keys_noalloc(at(0), n, 9, at(n), at(n + 1), None) == _capi.PBF_ERR_INVALID
    assert L.pbf_sort_keys_noalloc(at(0), n, 9, at(n - 1), at(3 * n), None) == _capi.PBF_ERR_INVALID
    assert b"overlap" in L.pbf_last_error()
    assert L.pbf_sort_keys_noalloc(at(0), (1 << 20) + 1, 9, at(n), at(2 * n), None) == _capi.PBF_ERR_INVALID
    assert b"exceed" in L.pbf_last_error()
    assert L.pbf_sort_keys_noalloc(at(0), n, 33, at(n), at(2 * n), None) == _capi.PBF_ERR_INVALID
    assert L.pbf_sort_keys_noalloc(None, n, 9, at(n), at(2 * n), None) == _capi.PBF_ERR_INVALID
    assert L.pbf_sort_keys_noalloc(at(0), 0, 9, at(0), at(0), None) == _capi.PBF_OK
