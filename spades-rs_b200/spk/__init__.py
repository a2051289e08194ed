"""spk -- Python view of libspk, the B200 k-mer counting library for spades-rs.

This package mirrors the reference's Rust interface for the counting path on
top of the C ABI in ``include/spk.h`` (loaded with ctypes from the in-tree
``libspk.so``):

* :class:`TwoTierFilter` -- ``TwoTierFilter`` of src/bloom.rs:13-131
  (``new``, ``insert``, ``is_solid``, ``insert_kmer256``, ``is_solid_kmer256``,
  ``memory_usage_bytes``), device resident, with batched forms.
* :func:`count` / :func:`count_solid_kmers` -- Stages 2-3 of
  ``run_assembly_with_packed_reads`` (src/assemble.rs:129-292) and the
  per-k loop of ``run_multik_assembly`` (src/multik.rs:109-178).
* :class:`Server` -- the serving loop (submit / poll / wait).

There is no CPU fallback: importing works anywhere, but every call that
needs the GPU raises :class:`SpkError` when ``libspk.so`` or the device is
missing.
"""
from ._lib import (SPK_F_CORRECT, SPK_F_DIRECT, SPK_F_EDGES, SPK_F_GATED, SPK_F_KEEP_BLOOM,
                   SPK_F_KEEP_TABLE, SPK_F_REF_SOLID,
                   SPK_SCHEDULE_COUNT_FIRST, SPK_SCHEDULE_FUSED, SPK_SCHEDULE_GATED,
                   SPK_SCHEDULE_PARTITIONED, SpkError, lib, lib_path, validate_k)
from .api import (Context, CountResult, DevicePackedReads, Job, PackedReads, Server, TwoTierFilter, count,
                  count_batch, count_batch_iter, count_device, count_solid_kmers, default_context, ingest, kmer256_from_limbs,
                  limbs_from_kmer256, nlimbs)

__all__ = [
    "SPK_F_CORRECT", "SPK_F_DIRECT", "SPK_F_EDGES", "SPK_F_GATED", "SPK_F_KEEP_BLOOM", "SPK_F_KEEP_TABLE",
    "SPK_F_REF_SOLID",
    "SPK_SCHEDULE_COUNT_FIRST", "SPK_SCHEDULE_FUSED", "SPK_SCHEDULE_GATED", "SPK_SCHEDULE_PARTITIONED",
    "SpkError", "lib", "lib_path",
    "validate_k", "Context", "CountResult", "DevicePackedReads", "Job", "PackedReads", "Server",
    "TwoTierFilter", "count", "count_batch", "count_batch_iter", "count_device", "count_solid_kmers", "default_context", "ingest",
    "kmer256_from_limbs", "limbs_from_kmer256", "nlimbs",
]
