"""fe_sort_pairs_noalloc: the radix sort that allocates no device memory.

Some callers cannot let the library allocate: a frame loop that must not
stall (cudaMalloc/cudaFree synchronise the device), work recorded by stream
capture in global mode, or a host that budgets all device memory itself.  For
them the sort's scratch is a static device array of the library.  This test
calls the entry point through the C ABI twice in a row, with different sizes
and key widths (so a stale scratch from the first call would show in the
second), and requires the same result as the allocating fe_sort_pairs, bit
for bit, as every sort test here does.  It lives in its own file, collected
last, and also passes alone in a fresh process (the first call sets up the
scratch address on the device).
"""
import ctypes

import numpy as np
import pytest

from fluid_step import _abi

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_sort_matches_allocating_sort_on_two_calls():
    import torch

    lib = _abi.load_library()
    torch.cuda.init()
    stream = torch.cuda.current_stream()
    cases = [(_abi.FE_SORT_NOALLOC_MAX_PAIRS, 32, 11),   # the maximum size, 4 passes
             (70_001, 20, 12)]                            # smaller, 3 passes, after it
    for n, key_bits, seed in cases:
        rng = np.random.default_rng(seed)
        keys = rng.integers(0, 1 << key_bits, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 3] = keys[0]                          # many equal keys: stability shows
        k_host = torch.from_numpy(keys.view(np.int32))
        v_host = torch.arange(n, dtype=torch.int32)
        ka, va = k_host.cuda(), v_host.cuda()
        kb, vb = k_host.cuda(), v_host.cuda()
        torch.cuda.synchronize()
        st = lib.fe_sort_pairs(_ptr(ka), _ptr(va), n, key_bits, _abi.FE_SORT_RADIX,
                               ctypes.c_void_p(stream.cuda_stream))
        assert st == _abi.FE_OK, lib.fe_last_error()
        st = lib.fe_sort_pairs_noalloc(_ptr(kb), _ptr(vb), n, key_bits,
                                       ctypes.c_void_p(stream.cuda_stream))
        assert st == _abi.FE_OK, lib.fe_last_error()
        torch.cuda.synchronize()
        assert torch.equal(ka, kb), "keys differ from fe_sort_pairs"
        assert torch.equal(va, vb), "values (the permutation) differ from fe_sort_pairs"
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(vb.cpu().numpy(), order.astype(np.int32))


def test_noalloc_sort_rejects_sizes_above_the_maximum():
    lib = _abi.load_library()
    st = lib.fe_sort_pairs_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16),
                                   _abi.FE_SORT_NOALLOC_MAX_PAIRS + 1, 32, None)
    assert st == _abi.FE_ERR_CAPACITY
    assert b"FE_SORT_NOALLOC_MAX_PAIRS" in lib.fe_last_error()
