"""Host side of the sharded multi-GPU count: which part of the work each rank
owns, the exchange of the twice tier, and the merge of the ranks' tables.

The reference counts on one host (src/assemble.rs:129-242).  Spread over G
ranks (one process per GPU, torch.distributed):

* Bloom.  Rank r owns the words [r W / G, (r + 1) W / G) of both tiers and
  applies the insert operations of every k-mer occurrence whose bit lies in
  them.  The seen and twice tiers do not depend on the order of the inserts
  (src/bloom.rs:95-97 with the twice tier), so the ranks' word ranges side by
  side are the single filter, bit for bit.  The twice tier is all-gathered
  (64 MiB at the default 512 Mi bits).
* Count.  Rank r owns the k-mers whose hash_kmer256(seed 1) lies in the r-th
  of G equal ranges of 2^64 -- a range of the count table's spans, since a
  span is the top bits of that hash.  It counts every occurrence of its own
  k-mers and admits a singleton when its three twice bits are set.  The
  ranks' tables are disjoint; the merged and sorted table is the single one.

Every rank takes the same collective steps in the same order.  The per-rank
compute is given as functions, so the same driver runs a rank's share on a
GPU or, in the tests, the oracle's restatement of it on the CPU.
"""
from __future__ import annotations

from typing import Callable, Tuple

import numpy as np


def word_range(num_words: int, rank: int, world: int) -> Tuple[int, int]:
    """Bloom words [lo, hi) owned by `rank`."""
    return num_words * rank // world, num_words * (rank + 1) // world


def owner(hash_seed1: np.ndarray, world: int) -> np.ndarray:
    """Owning rank of k-mers from their hash_kmer256(seed 1) values (uint64):
    floor(h * world / 2^64), in exact integer arithmetic (world < 2^31)."""
    h = np.asarray(hash_seed1, dtype=np.uint64)
    w = np.uint64(world)
    a, b = h >> np.uint64(32), h & np.uint64(0xFFFFFFFF)
    return ((a * w + ((b * w) >> np.uint64(32))) >> np.uint64(32)).astype(np.int32)


def _all_gather_u64(local: np.ndarray, sizes, group=None) -> list:
    """All-gather of variable-length uint64 arrays (as int64 tensors, padded)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    m = max(int(x) for x in sizes)
    buf = torch.zeros(max(m, 1), dtype=torch.int64)
    if local.size:
        buf[: local.size] = torch.from_numpy(np.ascontiguousarray(local).view(np.int64))
    outs = [torch.zeros(max(m, 1), dtype=torch.int64) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    return [o.numpy()[: int(n)].view(np.uint64).copy() for o, n in zip(outs, sizes)]


def gather_tier(local_words: np.ndarray, num_words: int, group=None) -> np.ndarray:
    """The whole tier from every rank's word range (all-gather)."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    lo, hi = word_range(num_words, rank, world)
    if local_words.size != hi - lo:
        raise ValueError(f"rank {rank} holds {local_words.size} words, owns {hi - lo}")
    sizes = [word_range(num_words, r, world)[1] - word_range(num_words, r, world)[0] for r in range(world)]
    return np.concatenate(_all_gather_u64(local_words, sizes, group))


def merge_tables(keys: np.ndarray, counts: np.ndarray, group=None) -> Tuple[np.ndarray, np.ndarray]:
    """Every rank's sorted (keys (n, L) uint64, counts uint32) merged into the
    sorted single table, on every rank (the ranks' keys are disjoint)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    L = keys.shape[1] if keys.ndim == 2 else 1
    n = torch.tensor([keys.shape[0]], dtype=torch.int64)
    ns = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(ns, n, group=group)
    sizes = [int(x.item()) for x in ns]
    kk = _all_gather_u64(np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1), [s * L for s in sizes], group)
    cc = _all_gather_u64(np.ascontiguousarray(counts, dtype=np.uint64), sizes, group)
    K = np.concatenate([k.reshape(-1, L) for k in kk]) if kk else np.zeros((0, L), np.uint64)
    Cn = np.concatenate(cc).astype(np.uint32)
    # Kmer256 order: limbs most significant last
    order = np.lexsort(tuple(K[:, j] for j in range(L))) if K.shape[0] else np.zeros(0, np.int64)
    return K[order], Cn[order]


def count_sharded(bloom_share: Callable[[int, int], Tuple[np.ndarray, np.ndarray]],
                  count_share: Callable[[np.ndarray, int, int], Tuple[np.ndarray, np.ndarray]],
                  num_words: int, group=None):
    """One sharded count.  bloom_share(rank, world) -> this rank's (seen,
    twice) words; count_share(twice, rank, world) -> this rank's sorted
    (keys, counts).  Returns (keys, counts, seen, twice) of the whole job on
    every rank."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    seen_l, twice_l = bloom_share(rank, world)
    twice = gather_tier(np.asarray(twice_l, dtype=np.uint64), num_words, group)
    seen = gather_tier(np.asarray(seen_l, dtype=np.uint64), num_words, group)
    keys, counts = count_share(twice, rank, world)
    K, Cn = merge_tables(keys, counts, group)
    return K, Cn, seen, twice
