"""spk_bloom_insert_k256_noalloc, the Bloom insert for callers that cannot
allocate device memory (their HBM is committed to their own arena or to
resident count tables, or they cannot take the device synchronisation an
allocation implies).  It is checked against spk_bloom_insert_k256, the
allocating entry point, through the C ABI, over two calls in a row so that
the second call runs on scratch that still holds the first call's contents.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _keys(rng, pool, n):
    """n Kmer256 keys drawn with repeats from pool (4 limbs each)."""
    return np.ascontiguousarray(pool[rng.integers(0, pool.shape[0], size=n)])


def test_noalloc_insert_matches_allocating_entry_point(spk_lib):
    import torch

    import spk
    from spk import _lib

    L = _lib.lib()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    ctx = spk.Context(0)
    bloom = spk.TwoTierFilter((1 << 20) + 37, ctx)  # rounded up to whole words
    words = bloom.size_bits // 64
    seen = torch.zeros(words, dtype=torch.int64, device=dev)
    solid = torch.zeros(words, dtype=torch.int64, device=dev)

    rng = np.random.default_rng(2024)
    # k = 55 keys: limbs 0-1 hold the 110-bit value, limbs 2-3 are zero.
    pool = np.zeros((40_000, 4), dtype=np.uint64)
    pool[:, 0] = rng.integers(0, 2 ** 63, size=40_000, dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=40_000, dtype=np.uint64)
    pool[:, 1] = rng.integers(0, 1 << 46, size=40_000, dtype=np.uint64)
    stream = torch.cuda.current_stream()

    for n in (_lib.SPK_NOALLOC_MAX_KEYS, 50_001):
        keys = _keys(rng, pool, n)
        want = bloom.insert_kmer256_batch(keys)
        d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
        d_prom = torch.full((n,), 7, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize()
        rc = L.spk_bloom_insert_k256_noalloc(seen.data_ptr(), solid.data_ptr(), words,
                                             d_keys.data_ptr(), n, d_prom.data_ptr(),
                                             C.c_void_p(stream.cuda_stream))
        assert rc == 0, _lib.last_error()
        stream.synchronize()
        got = d_prom.cpu().numpy().astype(bool)
        assert want.any() and not want.all()  # both outcomes occur
        np.testing.assert_array_equal(got, want)
        ref_seen, ref_solid = bloom.download()
        np.testing.assert_array_equal(seen.cpu().numpy().view(np.uint64), ref_seen)
        np.testing.assert_array_equal(solid.cpu().numpy().view(np.uint64), ref_solid)

    # More keys than the static scratch holds: refused with a clear error,
    # and nothing is written.
    before = seen.clone()
    n = _lib.SPK_NOALLOC_MAX_KEYS + 1
    d_keys = torch.zeros((n, 4), dtype=torch.int64, device=dev)
    rc = L.spk_bloom_insert_k256_noalloc(seen.data_ptr(), solid.data_ptr(), words,
                                         d_keys.data_ptr(), n, None, None)
    assert rc == 1 and "exceeds the maximum of 65536" in _lib.last_error()
    torch.cuda.synchronize()
    assert torch.equal(seen, before)
    bloom.close()
    ctx.close()
