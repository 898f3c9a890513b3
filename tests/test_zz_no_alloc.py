"""fe_sort_pairs_noalloc: the radix sort that allocates no device memory.

Some callers cannot let the library allocate: a frame loop that must not
stall (cudaMalloc/cudaFree synchronise the device), or a host that budgets
all device memory itself.  For
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


def _sort_noalloc(lib, n, seed, stream):
    import torch

    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    kd = torch.from_numpy(keys.view(np.int32)).cuda()
    vd = torch.arange(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = lib.fe_sort_pairs_noalloc(_ptr(kd), _ptr(vd), n, 32, ctypes.c_void_p(stream.cuda_stream))
    assert st == _abi.FE_OK, lib.fe_last_error()
    return keys, kd, vd


def _noalloc_flags(lib, stream):
    import torch

    word = ctypes.c_uint32(0xFFFFFFFF)
    st = lib.fe_sort_noalloc_flags(ctypes.byref(word), ctypes.c_void_p(stream.cuda_stream))
    assert st == _abi.FE_OK, lib.fe_last_error()
    torch.cuda.synchronize()
    return word.value


def test_noalloc_error_word_reports_a_wait_that_gave_up():
    """A sort whose bounded look-back wait gave up must not pass for a good
    one: the error word of the static array says so.  The test hook runs the
    same bounded wait on a word nothing publishes (no GPU fault), and the
    next sort clears the word again."""
    import torch

    lib = _abi.load_library()
    stream = torch.cuda.current_stream()
    keys, kd, vd = _sort_noalloc(lib, 5000, 21, stream)
    assert _noalloc_flags(lib, stream) == 0
    assert lib.fe_debug_noalloc_wait_timeout(1000, ctypes.c_void_p(stream.cuda_stream)) == 0
    assert _noalloc_flags(lib, stream) & _abi.FE_STATS_LOOKBACK_TIMEOUT
    keys, kd, vd = _sort_noalloc(lib, 5000, 22, stream)
    assert _noalloc_flags(lib, stream) == 0
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(vd.cpu().numpy(), order.astype(np.int32))
    # the flags can also land in device memory, in stream order
    dev_word = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    assert lib.fe_sort_noalloc_flags(_ptr(dev_word), ctypes.c_void_p(stream.cuda_stream)) == 0
    assert int(dev_word.item()) == 0


def test_allocating_sort_error_word_is_clear_after_a_good_sort():
    import torch

    lib = _abi.load_library()
    stream = torch.cuda.current_stream()
    n = 70_001
    kd = torch.randint(0, 1 << 20, (n,), dtype=torch.int32, device="cuda")
    vd = torch.arange(n, dtype=torch.int32, device="cuda")
    assert lib.fe_sort_pairs(_ptr(kd), _ptr(vd), n, 20, _abi.FE_SORT_RADIX,
                             ctypes.c_void_p(stream.cuda_stream)) == 0
    word = ctypes.c_uint32(0xFFFFFFFF)
    assert lib.fe_sort_flags(ctypes.byref(word), ctypes.c_void_p(stream.cuda_stream)) == 0
    torch.cuda.synchronize()
    assert word.value == 0


def test_noalloc_sort_takes_no_device_memory():
    """After a first call (which loads the kernels), a call leaves the
    device's free memory exactly as it was."""
    import torch

    lib = _abi.load_library()
    stream = torch.cuda.current_stream()
    n = 300_000
    _sort_noalloc(lib, n, 31, stream)
    torch.cuda.synchronize()
    rng = np.random.default_rng(32)
    kd = torch.from_numpy(rng.integers(0, 1 << 31, n).astype(np.int32)).cuda()
    vd = torch.arange(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = lib.fe_sort_pairs_noalloc(_ptr(kd), _ptr(vd), n, 32, ctypes.c_void_p(stream.cuda_stream))
    assert st == _abi.FE_OK, lib.fe_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
