"""next_sort_pairs_noalloc: the sort for callers that cannot allocate device memory.

Host codes that own every byte of device memory (a fixed per-GPU budget, their
own pool allocator) or that cannot pay for cudaMalloc/cudaFree synchronising
the device mid-step can only hand this library buffers they already own.  This
entry point sorts between such buffers and takes its scratch from a static
device array instead of allocating.  The test checks it against the
allocating entry point (next_sort_pairs, through a handle) bit for bit, on two
calls in a row so that scratch left by the first call cannot leak into the
second, and checks that it rejects sizes beyond its fixed maximum.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from next_b200 import native
from next_b200.native import Simulation

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1048576   # NEXT_SORT_NOALLOC_MAX_PAIRS


def _device_sort(lib, torch, keys, vals, key_bits):
    n = keys.shape[0]
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    ok = torch.empty_like(dk)
    ov = torch.empty_like(dv)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = lib.next_sort_pairs_noalloc(dk.data_ptr(), dv.data_ptr(), ok.data_ptr(), ov.data_ptr(), n, key_bits,
                                     torch.cuda.current_stream().cuda_stream)
    free_after = torch.cuda.mem_get_info()[0]
    assert rc == 0, native.load().next_status_string(rc)
    # the inputs are left as they were
    assert np.array_equal(dk.cpu().numpy().view(np.uint64), keys)
    return ok.cpu().numpy().view(np.uint64), ov.cpu().numpy().view(np.uint32), free_before - free_after


def test_noalloc_sort_matches_allocating_sort_on_two_calls():
    torch = pytest.importorskip("torch")
    lib = native.load()
    sim = Simulation("accurate", "mixed")
    cases = [(1_000_003, 63, 21), (MAX_PAIRS, 64, 22)]   # second call: different size and key width
    for call, (n, bits, seed) in enumerate(cases):
        rng = np.random.default_rng(seed)
        keys = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
        if bits == 64:
            keys |= rng.integers(0, 2, n, dtype=np.uint64) << np.uint64(63)
        keys[: n // 4] = keys[7]                      # long runs of equal keys: stability
        vals = rng.permutation(n).astype(np.uint32)
        want_k, want_v = sim.sort_pairs(keys, vals, bits)
        got_k, got_v, grown = _device_sort(lib, torch, keys, vals, bits)
        np.testing.assert_array_equal(got_k, want_k)
        np.testing.assert_array_equal(got_v, want_v)
        if call == 1:
            # set-up happened on the first call; later calls take no device memory
            assert grown == 0
    sim.close()


def test_noalloc_sort_rejects_oversize_and_aliasing():
    torch = pytest.importorskip("torch")
    lib = native.load()
    dk = torch.zeros(8, dtype=torch.int64, device="cuda")
    dv = torch.zeros(8, dtype=torch.int32, device="cuda")
    ok = torch.zeros(8, dtype=torch.int64, device="cuda")
    ov = torch.zeros(8, dtype=torch.int32, device="cuda")
    # larger than the static scratch: rejected before any device work
    assert lib.next_sort_pairs_noalloc(dk.data_ptr(), dv.data_ptr(), ok.data_ptr(), ov.data_ptr(),
                                       MAX_PAIRS + 1, 64, None) == 1
    # outputs may not alias the inputs
    assert lib.next_sort_pairs_noalloc(dk.data_ptr(), dv.data_ptr(), dk.data_ptr(), ov.data_ptr(), 8, 64, None) == 1
    assert lib.next_sort_pairs_noalloc(None, None, None, None, 0, 64, None) == 0
