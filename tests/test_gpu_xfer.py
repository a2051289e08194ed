"""Copies between pageable host memory and the device through the context's
pinned chunks (csrc/spk_xfer.cu): the reads a count uploads and the lists it
downloads are the same bytes whether the host buffers are pageable numpy
arrays (copied in 4 MiB pieces by several host threads) or pinned memory
(copied directly).  Integer data, compared bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def spk(spk_lib):
    return spk_lib


def pinned_copy(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


def test_pageable_and_pinned_uploads_agree(spk):
    """A read set of 38 MB (several upload pieces, each over the direct-copy
    size) counted from pageable and from pinned host buffers: same lists,
    edges and statistics; the downloads into pageable arrays equal those into
    pinned ones, and a piece-sized tail (not a multiple of the chunk) is
    whole."""
    from spk import synth
    p = synth.c2(0.3).packed
    assert p.data.size > 32 << 20
    hold = [pinned_copy(x) for x in (p.data, p.offsets, p.lengths)]
    pinned = tuple(h[1] for h in hold)
    a = spk.count(p, [31, 55], bloom_bits=1 << 28)
    b = spk.count(pinned, [31, 55], bloom_bits=1 << 28)
    for ki in range(2):
        ia, ib = a.info(ki), b.info(ki)
        for key in ("occurrences", "n_table", "n_list", "n_solid", "n_edges", "cutoff", "twice_popcount"):
            assert ia[key] == ib[key], key
        ka, ca = a.kmers(ki)
        kb, cb = b.kmers(ki)
        assert ka.nbytes > 8 << 20  # the download goes through the pinned chunks
        np.testing.assert_array_equal(ka, kb)
        np.testing.assert_array_equal(ca, cb)
        np.testing.assert_array_equal(a.edges(ki), b.edges(ki))
        # the same list into pinned output arrays
        m = ka.shape[0]
        tk, hk = pinned_copy(np.zeros((m + 3, ka.shape[1]), np.uint64))
        tc, hc = pinned_copy(np.zeros(m + 3, np.uint32))
        gk, gc = b.kmers(ki, out=(hk, hc))
        np.testing.assert_array_equal(gk, ka)
        np.testing.assert_array_equal(gc, ca)
    a.close()
    b.close()
