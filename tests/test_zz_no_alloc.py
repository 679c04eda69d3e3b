"""The allocation-free pair sort (mguso_radix_sort_pairs_noalloc) against the regular one.

Some hosts may not allocate device memory once they are running: an engine that hands the
whole GPU to its own memory pool at start-up, or a per-frame path that cannot pay for
cudaMalloc's device-wide synchronisation. The allocation-free entry point serves them from a
fixed scratch array inside the library; its output must equal mguso_radix_sort_pairs's
bit for bit. This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

import mguso
from mguso import _lib
from mguso.lbvh import NOALLOC_MAX_PAIRS, radix_sort_pairs, radix_sort_pairs_noalloc


def _pairs(rng, n, key_bits):
    if key_bits <= 32:
        # few distinct keys: long runs of equal keys test stability
        keys = rng.integers(0, 1 << min(key_bits, 12), n, dtype=np.uint64).astype(np.uint32)
    else:
        keys = rng.integers(0, 1 << key_bits, n, dtype=np.uint64)
        keys[rng.integers(0, n, n // 4)] = keys[0]
    vals = np.arange(n, dtype=np.uint32)
    return keys, vals


def test_noalloc_rejects_oversize_without_work():
    lib = _lib.load()
    rc = lib.mguso_radix_sort_pairs_noalloc(None, None, NOALLOC_MAX_PAIRS + 1, 30, None)
    assert rc == 1  # MGUSO_ERR_INVALID_ARG
    buf = C.create_string_buffer(256)
    lib.mguso_last_error(buf, 256)
    assert b"262144" in buf.value


@pytest.mark.gpu
@pytest.mark.parametrize("key_bits", [30, 63])
def test_noalloc_sort_equals_regular_sort_twice(key_bits):
    """Two calls in a row (different sizes, so the second one finds the first's leftovers in
    the shared scratch) each match the regular entry point exactly."""
    import torch

    ctx = mguso.Context(0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(key_bits)
    for n in (NOALLOC_MAX_PAIRS, 70001):
        keys, vals = _pairs(rng, n, key_bits)
        kt = torch.from_numpy(keys.view(np.int64) if keys.dtype == np.uint64 else keys.view(np.int32)).cuda()
        vt = torch.from_numpy(vals.view(np.int32)).cuda()
        k2, v2 = kt.clone(), vt.clone()
        torch.cuda.synchronize()
        radix_sort_pairs(ctx, kt.data_ptr(), vt.data_ptr(), n, key_bits, stream)
        radix_sort_pairs_noalloc(k2.data_ptr(), v2.data_ptr(), n, key_bits, stream)
        torch.cuda.synchronize()
        assert torch.equal(kt, k2) and torch.equal(vt, v2), n
        order = np.argsort(keys, kind="stable")
        got_k = k2.cpu().numpy().view(keys.dtype)
        assert np.array_equal(got_k, keys[order])
        assert np.array_equal(v2.cpu().numpy().view(np.uint32), vals[order])
    ctx.close()
