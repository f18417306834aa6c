"""next_sort_pairs_noalloc: the sort for callers that cannot allocate device memory.

Host codes that own every byte of device memory (a fixed per-GPU budget, their
own pool allocator) or that cannot pay for cudaMalloc/cudaFree synchronising
the device mid-step can only hand this library buffers they already own.  This
entry point sorts between such buffers and takes its scratch from a static
device array instead of allocating.  The tests check it bit for bit against
the allocating entry point (next_sort_pairs, through a handle) and against
NumPy's stable sort, on calls in a row so that scratch left by one call cannot
leak into the next: pass counts odd and even (key widths 8, 24, 63, 64 bits),
one and two pairs, and the fixed maximum size.  They also check that it
rejects sizes beyond that maximum and outputs that overlap an input.

This file is named to be collected last.
"""
import numpy as np
import pytest

from next_b200 import native
from next_b200.native import Simulation

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1048576   # NEXT_SORT_NOALLOC_MAX_PAIRS
INVALID = 1           # NEXT_ERR_INVALID_ARGUMENT


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
    assert np.array_equal(dv.cpu().numpy().view(np.uint32), vals)
    return ok.cpu().numpy().view(np.uint64), ov.cpu().numpy().view(np.uint32), free_before - free_after


def _case(n, bits, seed):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
    if bits == 64:
        keys |= rng.integers(0, 2, n, dtype=np.uint64) << np.uint64(63)
    if n > 8:
        keys[: n // 4] = keys[n // 2]               # long runs of equal keys: stability
    vals = rng.permutation(n).astype(np.uint32)
    return keys, vals


# (n, key_bits): 63 and 64 bits take 8 passes, 24 bits 3, 8 bits 1 (odd pass
# counts write the first pass straight into the outputs); n = 1 is a copy.
CASES = [(1_000_003, 63), (MAX_PAIRS, 64), (70_001, 24), (5_000, 8), (1, 64), (2, 24), (2, 8), (3840 * 3 + 1, 63)]


def test_noalloc_sort_matches_allocating_sort_on_calls_in_a_row():
    torch = pytest.importorskip("torch")
    lib = native.load()
    sim = Simulation("accurate", "mixed")
    for call, (n, bits) in enumerate(CASES):
        keys, vals = _case(n, bits, 21 + call)
        want_k, want_v = sim.sort_pairs(keys, vals, bits)
        got_k, got_v, grown = _device_sort(lib, torch, keys, vals, bits)
        np.testing.assert_array_equal(got_k, want_k)
        np.testing.assert_array_equal(got_v, want_v)
        # and against NumPy's stable sort of the significant bits
        mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
        order = np.argsort(keys & mask, kind="stable")
        np.testing.assert_array_equal(got_k, keys[order])
        np.testing.assert_array_equal(got_v, vals[order])
        if call >= 1:
            # set-up happened on the first call; later calls take no device memory
            assert grown == 0
    sim.close()


def test_noalloc_sort_rejects_oversize_and_overlap():
    torch = pytest.importorskip("torch")
    lib = native.load()
    dk = torch.zeros(64, dtype=torch.int64, device="cuda")
    dv = torch.zeros(64, dtype=torch.int32, device="cuda")
    ok = torch.zeros(64, dtype=torch.int64, device="cuda")
    ov = torch.zeros(64, dtype=torch.int32, device="cuda")
    k, v, o, w = dk.data_ptr(), dv.data_ptr(), ok.data_ptr(), ov.data_ptr()
    # larger than the static scratch: rejected before any device work
    assert lib.next_sort_pairs_noalloc(k, v, o, w, MAX_PAIRS + 1, 64, None) == INVALID
    # outputs may not overlap an input or each other, in whole or in part
    assert lib.next_sort_pairs_noalloc(k, v, k, w, 8, 64, None) == INVALID
    assert lib.next_sort_pairs_noalloc(k, v, o, v, 8, 64, None) == INVALID
    assert lib.next_sort_pairs_noalloc(k, v, k + 8 * 4, w, 8, 64, None) == INVALID      # keys_out inside keys_in
    assert lib.next_sort_pairs_noalloc(k, v, o, k + 16, 8, 64, None) == INVALID         # vals_out inside keys_in
    assert lib.next_sort_pairs_noalloc(k, v, o, o + 8 * 7, 8, 64, None) == INVALID      # vals_out inside keys_out
    assert lib.next_sort_pairs_noalloc(k, v, o, w, 8, 0, None) == INVALID
    assert lib.next_sort_pairs_noalloc(None, None, None, None, 0, 64, None) == 0
    # adjacent but disjoint buffers are fine
    assert lib.next_sort_pairs_noalloc(k, v, k + 8 * 8, w, 8, 64, None) == 0
