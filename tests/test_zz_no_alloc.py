"""The sort entry point that allocates nothing (hmg_radix_sort_u64_noalloc).

Some callers of this library cannot let it call cudaMalloc: a host program that
hands all device memory to its own pool at start-up, or a latency-bound loop where
an allocation (and the device synchronisation it implies) is not acceptable.  The
no-allocation variant sorts with a fixed scratch array compiled into the library
instead.  This test drives it through the C ABI, twice in a row with different
inputs (the scratch keeps the previous call's contents), and requires the exact
result of the allocating entry point hmg_radix_sort_u64.  It lives in its own file,
collected last, and passes both alone and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20


def _sorted_pair(torch, fn, keys, vals, key_bits):
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    torch.cuda.synchronize()
    st = fn(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), keys.shape[0], key_bits, None)
    torch.cuda.synchronize()
    return st, dk.cpu().numpy().view(np.uint64), dv.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort(hmg, cuda):
    torch = cuda
    L = hmg.lib()
    noalloc = L.hmg_radix_sort_u64_noalloc
    noalloc.restype = C.c_int
    noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    rng = np.random.default_rng(2024)
    # calls in a row: Morton-like 60-bit keys with repeats (the two low digits are
    # the same for every key, so those passes are skipped on the device), full 64-bit
    # keys, then keys that are all equal (every pass skipped) on a ragged last tile
    cases = [(MAX_KEYS, 60, 1 << 40), (300007, 64, None), (5000, 64, 1)]
    for n, key_bits, distinct in cases:
        if distinct == 1:
            keys = np.full(n, 0x0123456789ABCDEF, dtype=np.uint64)
        elif distinct is None:
            keys = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) | (
                rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63))
        else:
            keys = rng.integers(0, distinct, size=n, dtype=np.uint64) << np.uint64(20)
        vals = np.arange(n, dtype=np.uint32)
        st_a, ka, va = _sorted_pair(torch, L.hmg_radix_sort_u64, keys, vals, key_bits)
        st_b, kb, vb = _sorted_pair(torch, noalloc, keys, vals, key_bits)
        assert st_a == 0 and st_b == 0, L.hmg_last_error()
        np.testing.assert_array_equal(kb, ka)
        np.testing.assert_array_equal(vb, va)
        assert np.all(ka[1:] >= ka[:-1])
    # beyond the fixed capacity: rejected with a clear message, inputs untouched
    big = np.zeros(1, dtype=np.uint64)
    dk = torch.from_numpy(big.view(np.int64)).cuda()
    st = noalloc(C.c_void_p(dk.data_ptr()), C.c_void_p(dk.data_ptr()), MAX_KEYS + 1, 64, None)
    assert st == 1
    assert b"capacity" in L.hmg_last_error()
