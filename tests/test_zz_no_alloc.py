"""GPU test of gsplat_cuda_sort_values_by_keys_noalloc, the sort for callers
that cannot allocate device memory (hosts that own all GPU memory through
their own pool, or latency-critical threads where cudaMalloc/cudaFree are not
allowed). The caller brings device buffers; the sort's scratch comes from a
static device array inside the library.

The test owns its device buffers (allocated here with torch, as such a host
would from its own pool), calls the entry point through the C ABI twice in a
row with different data and lengths — the second call must not see the first
call's leftovers in the shared scratch — and checks both results bit for bit
(sorting is exact integer work, so the tolerance is zero) against the
allocating gsplat_cuda_sort_values_by_keys and against the oracle's
restatement of the reference sort (CpuSortBackend::sort_values_by_keys,
crates/gsplat-sort/src/lib.rs:36-61). The file sorts last so that a run
stopping at its first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

import gsplat_ffi as ffi

pytestmark = pytest.mark.gpu

MAX_ITEMS = 1 << 20


def _noalloc_sort(keys, values):
    import torch

    dk = torch.from_numpy(keys.view(np.int32).copy()).cuda()
    dv = torch.from_numpy(values.view(np.int32).copy()).cuda()
    torch.cuda.synchronize()
    rc = ffi.lib().gsplat_cuda_sort_values_by_keys_noalloc(
        ctypes.c_void_p(dk.data_ptr()), ctypes.c_void_p(dv.data_ptr()), len(keys), None)
    ffi.check(rc)
    torch.cuda.synchronize()
    out_keys = dk.cpu().numpy().view(np.uint32)
    out_vals = dv.cpu().numpy().view(np.uint32)
    return out_keys, out_vals


def test_noalloc_sort_matches_allocating_sort_twice(oracle):
    rng = np.random.default_rng(2024)
    # First call: near the limit, heavy key ties (the tie order is the part a
    # stale scratch or a wrong buffer hand-over would break first).
    n1 = MAX_ITEMS - 3
    k1 = rng.integers(0, 1 << 12, n1, dtype=np.uint32)
    v1 = rng.permutation(n1).astype(np.uint32)
    got_k1, got_v1 = _noalloc_sort(k1, v1)
    assert np.array_equal(got_k1, k1), "keys must be left unchanged"
    assert np.array_equal(got_v1, ffi.sort_values_by_keys(k1, v1))
    assert np.array_equal(got_v1, oracle.sort_values_by_keys(k1, v1))
    # Second call: shorter, different key distribution, on the same scratch.
    n2 = 70001
    k2 = rng.integers(0, 1 << 32, n2, dtype=np.uint64).astype(np.uint32)
    k2[::7] = 0xFFFFFFFF
    v2 = np.arange(n2, dtype=np.uint32)
    got_k2, got_v2 = _noalloc_sort(k2, v2)
    assert np.array_equal(got_k2, k2)
    assert np.array_equal(got_v2, ffi.sort_values_by_keys(k2, v2))
    assert np.array_equal(got_v2, oracle.sort_values_by_keys(k2, v2))


def test_noalloc_sort_rejects_lengths_above_the_limit():
    rc = ffi.lib().gsplat_cuda_sort_values_by_keys_noalloc(None, None, MAX_ITEMS + 1, None)
    assert rc == ffi.INVALID_ARGUMENT
    assert "exceeds the no-allocation limit" in ffi.last_error()


def test_noalloc_sort_refuses_a_capturing_stream():
    """The call synchronises its stream, which would invalidate a capture in
    progress: it must refuse the stream and leave the capture intact."""
    import torch

    keys = torch.zeros(1024, dtype=torch.int32, device="cuda")
    vals = torch.arange(1024, dtype=torch.int32, device="cuda")
    # first call outside any capture (sets up the device's scratch address)
    ffi.check(ffi.lib().gsplat_cuda_sort_values_by_keys_noalloc(
        ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(vals.data_ptr()), 1024, None))
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        rc = ffi.lib().gsplat_cuda_sort_values_by_keys_noalloc(
            ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(vals.data_ptr()), 1024,
            ctypes.c_void_p(stream.cuda_stream))
        vals.add_(1)  # the capture must still be valid after the refusal
    assert rc == ffi.INVALID_ARGUMENT
    assert "captured" in ffi.last_error()
    graph.replay()
    torch.cuda.synchronize()
    assert int(vals[0].item()) == 1
