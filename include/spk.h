/*
 * spk.h -- C ABI of libspk, the B200 (sm_100a) k-mer counting library for the
 * spades-rs assembler.
 *
 * The library replaces the k-mer counting hot path of spades-rs:
 *   - the two-tier Bloom prefilter    (src/bloom.rs:13-131, TwoTierFilter),
 *   - Stage 2 Bloom population        (src/assemble.rs:129-161),
 *   - Stage 3 solid k-mer count table (src/assemble.rs:166-242),
 *   - the solid-k-mer cutoff and set  (src/assemble.rs:286-292, 692-735),
 *   - (k+1)-mer edges implied by      (src/graph.rs:78-102),
 *   - the per-k loop of multi-k runs  (src/multik.rs:109-178),
 * and the steps either side of it:
 *   - FASTQ / FASTA ingest into the PackedReads store (src/packed_reads.rs:69-690),
 *   - single-base read error correction (src/hammer.rs:34-121) and the
 *     correcting Stage 3 (src/assemble.rs:183-191),
 *   - the prior-contig boost          (src/assemble.rs:244-284),
 *   - unitig compaction               (src/graph.rs:65-235).
 * The reference computes all of this on host threads; here everything runs on
 * one GPU and the host only moves buffers across this boundary.
 *
 * Conventions
 *   - Every call returns an int status; SPK_OK (0) is success.  On failure
 *     spk_last_error() returns a message for the calling thread.  No call
 *     aborts the process.
 *   - k-mer keys are passed as little-endian u64 limbs of the reference
 *     Kmer256 (src/dna.rs:134-138): limb 0 = lo bits 0..63, limb 1 = lo bits
 *     64..127, limb 2 = hi bits 0..63, limb 3 = hi bits 64..127.  Lists of
 *     k-mers use ceil(k/32) limbs per key; "k256" entry points always use 4.
 *   - Lists are sorted ascending in Kmer256 order (lexicographic on (lo, hi),
 *     src/dna.rs:137), which is sequence order for a fixed k.
 *   - Input host buffers are borrowed for the duration of a call.  Results
 *     are owned by the library until spk_result_free.
 *   - A context may be used from one host thread at a time, except the
 *     spk_submit / spk_poll / spk_wait family, which is thread-safe.
 *   - The packed read layout is the reference PackedReads store
 *     (src/packed_reads.rs:42-59, 547-578): 2 bits per base, A=0 C=1 G=2 T=3,
 *     first base in the two most significant bits of a byte, every read
 *     starting on a byte boundary at offsets[i] with lengths[i] bases.
 */
#ifndef SPK_H
#define SPK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPK_VERSION 1

/* Status codes. */
enum spk_status {
  SPK_OK = 0,
  SPK_E_INVALID_ARG = 1,  /* null pointer, size mismatch, read out of bounds */
  SPK_E_INVALID_K = 2,    /* k outside the supported range (src/main.rs:11-30) */
  SPK_E_OOM = 3,          /* device memory exhausted */
  SPK_E_TABLE_FULL = 4,   /* count table overflowed after regrow attempts */
  SPK_E_TIMEOUT = 5,      /* a bounded device-side wait expired */
  SPK_E_CUDA = 6,         /* CUDA runtime error */
  SPK_E_NO_DEVICE = 7,    /* no usable sm_100 device */
  SPK_E_ADMISSION = 8,    /* serving: job can never fit the HBM budget */
  SPK_E_NOT_READY = 9,    /* serving: job not finished within the wait */
  SPK_E_NOT_FOUND = 10    /* serving: unknown ticket */
};

typedef struct spk_ctx spk_ctx;
typedef struct spk_bloom spk_bloom;
typedef struct spk_result spk_result;

/* Message of the last failed call on this thread ("" if none). */
const char* spk_last_error(void);
int spk_version(void);

/* The CLI rule for k (src/main.rs:11-30): odd and in 11..=127.  Returns
 * SPK_OK or SPK_E_INVALID_K with the reference's wording in spk_last_error().
 * spk_count itself accepts any 1 <= k <= 127, as src/dna.rs does. */
int spk_validate_k(uint32_t k);

/* ---- context ------------------------------------------------------------ */
int spk_ctx_create(int device, spk_ctx** out);
int spk_ctx_destroy(spk_ctx* ctx);
/* Device memory currently held by the context's pools, in bytes. */
int spk_ctx_memory(spk_ctx* ctx, uint64_t* reserved_bytes, uint64_t* free_bytes);
/* Runs the context's work on a caller-owned cudaStream_t (NULL restores the
 * context's own stream), so callers can order libspk work with their own
 * kernels and time it with events on that stream. */
int spk_ctx_set_stream(spk_ctx* ctx, void* cuda_stream);

/* ---- TwoTierFilter (src/bloom.rs:13-131) --------------------------------
 * A device-resident two-tier Bloom filter with the reference's bit layout,
 * hash (src/bloom.rs:61-78) and seeds (src/bloom.rs:84-86).  Batched calls
 * have exactly the result of calling the reference method once per key in
 * array order. */
/* TwoTierFilter::new (src/bloom.rs:26-43): rounds capacity up to 64-bit words. */
int spk_bloom_create(spk_ctx* ctx, uint64_t capacity_bits, spk_bloom** out);
int spk_bloom_destroy(spk_bloom* bloom);
/* size_bits of src/bloom.rs:15 and memory_usage_bytes of src/bloom.rs:129-131. */
uint64_t spk_bloom_size_bits(const spk_bloom* bloom);
uint64_t spk_bloom_memory_usage_bytes(const spk_bloom* bloom);
/* TwoTierFilter::insert (src/bloom.rs:48-50), one key per element.
 * out_promoted[i] (nullable) = the bool the reference returns. */
int spk_bloom_insert_u64(spk_bloom* bloom, const uint64_t* keys, size_t n, uint8_t* out_promoted);
/* TwoTierFilter::insert_kmer256 (src/bloom.rs:83-107); keys are 4 limbs each. */
int spk_bloom_insert_k256(spk_bloom* bloom, const uint64_t* keys4, size_t n, uint8_t* out_promoted);
/* TwoTierFilter::is_solid (src/bloom.rs:54-56). */
int spk_bloom_is_solid_u64(spk_bloom* bloom, const uint64_t* keys, size_t n, uint8_t* out);
/* TwoTierFilter::is_solid_kmer256 (src/bloom.rs:111-126). */
int spk_bloom_is_solid_k256(spk_bloom* bloom, const uint64_t* keys4, size_t n, uint8_t* out);
/* Copy the tiers (seen_bits / solid_bits of src/bloom.rs:19-21) to the host;
 * each buffer holds size_bits/64 words and may be NULL. */
int spk_bloom_download(spk_bloom* bloom, uint64_t* seen, uint64_t* solid);

/* Largest n accepted by spk_bloom_insert_k256_noalloc. */
#define SPK_NOALLOC_MAX_KEYS 65536u
/* No counterpart in the reference.  The insert_kmer256 batch of
 * spk_bloom_insert_k256 for callers that must not allocate device memory:
 * hosts whose HBM is fully committed to their own arena or to resident count
 * tables (a cudaMalloc would fail there), and hosts with work in flight on
 * other streams that cannot afford the implicit device synchronisation of
 * cudaMalloc / cudaFree.  Everything is a device pointer on the current
 * device and owned by the caller: the two tiers (num_words u64 words each,
 * size_bits = 64 * num_words as in src/bloom.rs:27-28), n keys of 4 limbs and
 * the nullable out_promoted (n bytes).  The result equals
 * spk_bloom_insert_k256 on a filter holding the same tiers.
 *   - n may be at most SPK_NOALLOC_MAX_KEYS; larger n returns
 *     SPK_E_INVALID_ARG and does nothing.
 *   - The work is queued on cuda_stream (NULL = the legacy default stream)
 *     and the call returns without waiting; the outputs are ready once that
 *     stream has been synchronised.
 *   - The library never allocates for this call.  Its scratch (about 10 MiB)
 *     is a static device array that every GPU holds from the moment the
 *     library's device code is loaded on it until the process exits.
 *   - The first call on each device looks up that array's device address;
 *     make that first call before any stream capture on the device.
 *   - All calls on a device share the one scratch array, so calls whose work
 *     overlaps on the GPU (different streams, or different host threads
 *     without ordering) race and give wrong results: order them on one
 *     stream or synchronise between them. */
int spk_bloom_insert_k256_noalloc(uint64_t* d_seen, uint64_t* d_solid, uint64_t num_words,
                                  const uint64_t* d_keys4, size_t n, uint8_t* d_out_promoted,
                                  void* cuda_stream);

/* ErrorCorrector::correct_read_in_place (src/hammer.rs:34-121) on every read
 * of a packed read set, against this filter's solid tier, as Stage 3 applies
 * it before counting (src/assemble.rs:183-191).  data_out (data_len bytes;
 * may equal data) receives the packed data with the corrected bases in place;
 * reads shorter than k are unchanged.  corrected (nullable, n_reads bytes)
 * gets 1 for every read with a changed base, *n_corrected (nullable) their
 * number.  k: 0 corrects nothing (as the reference); 1..127; reads of at most
 * 8192 bases (longer ones: SPK_E_INVALID_ARG).  The result equals calling the
 * reference once per read in any order (reads are independent). */
int spk_bloom_correct_reads(spk_bloom* bloom, uint32_t k, const uint8_t* data, size_t data_len,
                            const uint64_t* offsets, const uint32_t* lengths, size_t n_reads,
                            uint8_t* data_out, uint8_t* corrected, uint64_t* n_corrected);
/* The same on device-resident reads: every pointer except n_corrected is a
 * device pointer on the filter's device. */
int spk_bloom_correct_reads_device(spk_bloom* bloom, uint32_t k, const uint8_t* d_data, size_t data_len,
                                   const uint64_t* d_offsets, const uint32_t* d_lengths, size_t n_reads,
                                   uint8_t* d_data_out, uint8_t* d_corrected, uint64_t* n_corrected);

/* ---- FASTQ / FASTA ingest (src/packed_reads.rs:69-690) ------------------
 * PackedReads::from_paired_files (text2 != NULL) or append_from_file into an
 * empty store (text2 == NULL) over decompressed FASTQ or FASTA texts (each
 * text is detected on its own, as FastxReader::open does; gzip stays with the
 * caller, as flate2 does in the reference).  The three gates and the
 * three-block layout (src/packed_reads.rs:8-27): terminal N trim, pairs
 * whose trimmed mates both have no internal N and MIN_K (21) bases or more
 * go to Block 1 (R1) and Block 2 (R2), the N-split sub-reads of MIN_K bases
 * or more of every other record go to Block 3, and records with no such
 * sub-read go to the ambiguous sidecar.  The store stays on the device
 * (spk_packed_device gives pointers for spk_count_device).  Malformed texts
 * return SPK_E_INVALID_ARG with the reference's message.  Each text must be
 * shorter than 4 GiB. */
typedef struct spk_packed spk_packed;
int spk_ingest(spk_ctx* ctx, const uint8_t* text1, size_t len1, const uint8_t* text2, size_t len2,
               spk_packed** out);
int spk_packed_info(const spk_packed* p, uint64_t* n_reads, uint64_t* data_len, uint64_t* pe_count,
                    uint64_t* n_sidecar, uint64_t* sidecar_bytes);
/* Device time of the ingest (text upload included) and its kernel launches. */
int spk_packed_stats(const spk_packed* p, float* ms_device, uint32_t* kernel_launches);
/* Host copies: data (data_len bytes), offsets / lengths (n_reads each), the
 * sidecar reads concatenated (sidecar_bytes) and their lengths (n_sidecar).
 * Any pointer may be NULL. */
int spk_packed_download(spk_packed* p, uint8_t* data, uint64_t* offsets, uint32_t* lengths,
                        uint8_t* sidecar, uint64_t* sidecar_lengths);
/* Device pointers of the store (valid until spk_packed_free); data is padded
 * for spk_count_device. */
int spk_packed_device(spk_packed* p, const uint8_t** d_data, const uint64_t** d_offsets,
                      const uint32_t** d_lengths);
int spk_packed_free(spk_packed* p);

/* ---- counting (src/assemble.rs:129-292, src/graph.rs:78-102) ------------ */
#define SPK_F_EDGES      0x1u  /* build the (k+1)-mer edge list */
#define SPK_F_REF_SOLID  0x2u  /* also build the reference-semantics solid tier */
#define SPK_F_KEEP_BLOOM 0x4u  /* keep the Bloom tiers for spk_result_bloom */
#define SPK_F_GATED      0x8u  /* the reference's two-pass schedule: Stage 3 counts only
                                  occurrences admitted by the final Bloom.  Same result as
                                  the default one-pass schedules (which count every k-mer
                                  and admit singletons afterwards) with a table that holds
                                  only admitted k-mers, for read sets too large for that */
#define SPK_F_DIRECT     0x10u /* count-first with one global-table atomic per occurrence
                                  instead of the partitioned passes */
#define SPK_F_CORRECT    0x20u /* Stage 3 with error correction (config.error_correct,
                                  src/assemble.rs:183-191): after the Bloom pass every read
                                  is corrected against the twice tier (src/hammer.rs:34-121)
                                  into a device copy, and the count pass reads the
                                  corrected copy.  Implies SPK_F_GATED. */
#define SPK_F_KEEP_TABLE 0x40u /* keep the count table for spk_result_table_view.  Without it
                                  the partitioned schedule writes the k-mer list directly
                                  from its spans and never materialises the table, and the
                                  other schedules (and prior contigs), which need it while
                                  counting, free it when the job ends */

/* spk_result_info.schedule */
#define SPK_SCHEDULE_GATED       0u  /* SPK_F_GATED: Bloom pass, then the gated count pass */
#define SPK_SCHEDULE_FUSED       1u  /* SPK_F_REF_SOLID: one read pass with the per-occurrence
                                        Bloom inserts the reference solid tier needs */
#define SPK_SCHEDULE_COUNT_FIRST 2u  /* one read pass counting every k-mer into the table with
                                        global atomics (SPK_F_DIRECT; k = 96; k > 64 on read sets
                                        too small for two partition levels); the Bloom tiers are
                                        derived from the table afterwards */
#define SPK_SCHEDULE_PARTITIONED 3u  /* the default: the read pass scatters keys by table span,
                                        each span is counted in shared memory and written once,
                                        with the Bloom tiers derived from its counts */

typedef struct spk_count_opts {
  uint64_t bloom_bits;    /* bits per tier; 0 = 512 Mi (src/assemble.rs:84) */
  uint32_t min_count;     /* 0 = adaptive cutoff (src/assemble.rs:692-735), else fixed */
  uint32_t list_min_count;/* smallest count kept in the sorted k-mer list (default 2) */
  double min_coverage;    /* min_coverage of the adaptive cutoff (default 5.0) */
  uint32_t flags;         /* SPK_F_* (default SPK_F_EDGES | SPK_F_KEEP_BLOOM) */
  uint32_t table_log2;    /* 0 = size the count table automatically; else start with
                             2^table_log2 slots (it still grows on overflow) */
  /* Prior and trusted contigs (src/assemble.rs:244-284): ASCII sequences in
   * host memory, contig i = prior_seqs[prior_offsets[i] .. + prior_lengths[i]),
   * borrowed for the call (for spk_job: until the job completes).  Every
   * k-window of a contig that Kmer256::from_bytes accepts (src/dna.rs:299-321)
   * adds max(4 * (uint32_t)min_coverage, 50) to its canonical k-mer's count,
   * after singleton admission and before the cutoff; a k-mer the table does
   * not hold is inserted with that count.  n_prior = 0: none. */
  const uint8_t* prior_seqs;
  const uint64_t* prior_offsets;
  const uint32_t* prior_lengths;
  uint64_t n_prior;
  uint32_t span_groups_log2;  /* default job: count in at least 2^span_groups_log2 groups of spans
                                 (one pass over the reads each); 0 = as many as the device
                                 memory needs (usually one) */
  uint32_t reserved;
  /* Host buffers (pageable or pinned; either may be NULL) that receive the
   * solid list of the first k, as spk_result_solid gives it, during the count:
   * the default job copies it while the edges are built.  solid_capacity is
   * the k-mers they hold (keys: ceil(k/32) limbs each); a longer list is not
   * copied.  spk_result_info.solid_copied tells whether they were filled, and
   * n_solid how many k-mers they hold.  Borrowed for the call. */
  uint64_t* solid_keys_out;
  uint32_t* solid_counts_out;
  uint64_t solid_capacity;
} spk_count_opts;

void spk_count_opts_default(spk_count_opts* opts);

/* Counts canonical k-mers of the packed reads for each k in ks[0..n_k).
 * Replaces Stages 2-3 of run_assembly_with_packed_reads
 * (src/assemble.rs:122-292) for one k, and the per-k loop of
 * run_multik_assembly (src/multik.rs:109-178) for several.  Host buffers are
 * copied to the device inside the call. */
int spk_count(spk_ctx* ctx, const uint8_t* data, size_t data_len, const uint64_t* offsets,
              const uint32_t* lengths, size_t n_reads, const uint32_t* ks, int n_k,
              const spk_count_opts* opts, spk_result** out);
/* Same with the packed reads already resident on the context's device.
 * d_data must have data_len + 64 readable bytes (the tail is ignored). */
int spk_count_device(spk_ctx* ctx, const uint8_t* d_data, size_t data_len,
                     const uint64_t* d_offsets, const uint32_t* d_lengths, size_t n_reads,
                     const uint32_t* ks, int n_k, const spk_count_opts* opts, spk_result** out);

typedef struct spk_result_info {
  uint32_t k;
  uint32_t cutoff;               /* solid threshold used (src/assemble.rs:286) */
  uint64_t occurrences;          /* k-mer positions per pass */
  uint64_t admitted_occurrences; /* positions admitted to the table */
  uint64_t n_table;              /* distinct admitted k-mers (the HashMap's len) */
  uint64_t n_list;               /* k-mers with count >= list_min_count */
  uint64_t n_solid;              /* k-mers with count >= cutoff */
  uint64_t n_edges;              /* canonical (k+1)-mer edges */
  uint64_t n_singletons;         /* admitted k-mers with count 1 */
  uint64_t bloom_size_bits;
  uint64_t seen_popcount;
  uint64_t twice_popcount;
  uint64_t table_capacity;
  uint32_t table_regrows;
  uint32_t kernel_launches;      /* libspk kernels launched for this k */
  float ms_bloom, ms_count, ms_finish, ms_sort, ms_edges, ms_total; /* device time per phase */
  float ms_bloom_kernel;         /* the kernel that fills the Bloom tiers */
  float ms_count_kernel;         /* the count kernel alone (last attempt; 0 for the fused
                                    schedule, whose one kernel is ms_bloom_kernel; the span
                                    count for the partitioned schedule) */
  uint32_t schedule;             /* SPK_SCHEDULE_* */
  uint32_t part_rescatters;      /* partitioned: read passes repeated with exact region sizes */
  uint64_t n_distinct;           /* distinct k-mers in the table before singleton admission
                                    (n_table plus the rejected singletons) */
  float ms_scatter_kernel;       /* partitioned: the read pass that scatters keys by span */
  float ms_unitigs;              /* spk_result_unitigs: device time of the build, through the
                                    copy of the unitigs to the host (0 until built) */
  float ms_unitigs_host;         /* ... and the host's orientation and sort of the unitigs */
  uint32_t unitig_launches;      /* kernels the unitig build launched */
  uint64_t n_unitigs;
  uint64_t n_corrected_reads;    /* SPK_F_CORRECT: reads with a corrected base */
  float ms_correct;              /* SPK_F_CORRECT: device time of the correction */
  uint32_t part_passes;          /* partitioned: 1 = the keys went to their spans in one pass,
                                    2 = through coarse buckets first (ms_scatter_kernel covers
                                    both passes) */
  uint32_t span_groups;          /* partitioned: passes over the reads, each partitioning and
                                    counting one group of spans (read sets too large for one) */
  float ms_coarse_kernel;        /* two-level partition in one group: the coarse pass alone
                                    (ms_scatter_kernel - ms_coarse_kernel is the fine pass) */
  uint32_t solid_copied;         /* 1: the solid list went to spk_count_opts.solid_*_out */
  uint32_t reserved2;
} spk_result_info;

int spk_result_count(const spk_result* res, int* n_k);
int spk_result_info_get(const spk_result* res, int k_index, spk_result_info* info);
/* Solid k-mers (count >= cutoff), sorted.  *n_inout: capacity in, count out.
 * keys_out gets ceil(k/32) limbs per key; either output may be NULL to query n. */
int spk_result_solid(spk_result* res, int k_index, uint64_t* keys_out, uint32_t* counts_out,
                     size_t* n_inout);
/* Sorted (k-mer, count) list of every k-mer with count >= max(min_count, list_min_count). */
int spk_result_kmers(spk_result* res, int k_index, uint32_t min_count, uint64_t* keys_out,
                     uint32_t* counts_out, size_t* n_inout);
/* Canonical (k+1)-mer edges, sorted, ceil((k+1)/32) limbs each. */
int spk_result_edges(spk_result* res, int k_index, uint64_t* edges_out, size_t* n_inout);
/* Bloom tiers of the count: seen (bit-exact with src/bloom.rs:95-97), the
 * twice tier, and the reference-semantics solid tier (SPK_F_REF_SOLID).  Each
 * buffer holds bloom_size_bits/64 words and may be NULL. */
int spk_result_bloom(spk_result* res, int k_index, uint64_t* seen, uint64_t* twice,
                     uint64_t* ref_solid);

/* Device-resident count table for a downstream graph build on the same
 * device (the input of CompactedGraph::build, src/graph.rs:65-69).  Open
 * addressing with linear probing from slot h = hash_kmer256(key, seed 1) >>
 * (64 - log2(capacity)) (src/bloom.rs:61-78, seed src/bloom.rs:84); the
 * table is divided into spans of 2^log2span slots and the probe sequence
 * wraps inside the span holding h: slot i of the sequence is
 * (h & ~(span - 1)) | ((h + i) & (span - 1)).  Slot s
 * starts at slots + s * slot_bytes with key_limbs u64 key limbs, followed by
 * a u32 count at byte key_limbs * 8: 0 = empty, bit 31 set = a k-mer seen
 * once that the Bloom did not admit.  Valid until spk_result_free. */
typedef struct spk_table_view {
  const void* slots;      /* device pointer */
  uint64_t capacity;
  uint32_t key_limbs;     /* ceil(k/32) */
  uint32_t slot_bytes;
  uint32_t k;
  uint32_t cutoff;
  uint32_t log2span;      /* probe sequences wrap inside spans of 2^log2span slots */
  uint32_t reserved;
  /* Keys are stored as the 2k-bit sequence value (first base most
   * significant), little-endian limbs.  For k <= 64 that equals the Kmer256
   * limbs; for k > 64 the Kmer256 form is (value >> 2(k-64), value & mask). */
} spk_table_view;
/* Fails with SPK_E_INVALID_ARG when the job did not keep the table (counted
 * without SPK_F_KEEP_TABLE). */
int spk_result_table_view(spk_result* res, int k_index, spk_table_view* view);

/* Unitigs of the solid k-mers: the maximal non-branching paths of their de
 * Bruijn graph, one per reverse-complement pair, as CompactedGraph::build
 * (src/graph.rs:65-235) finds them.  An isolated cycle is cut at its smallest
 * solid k-mer read forward, where the reference's walk in sorted order starts.
 * Replaces the unitig list of CompactedGraph (src/graph.rs:44-62); the Rust
 * side orders its unitigs by hash-set iteration, so here each unitig is
 * given in the orientation not greater than its reverse complement and the
 * list is sorted by sequence.  k must be odd (src/main.rs:10-23).
 *
 * seqs receives the concatenated ASCII sequences (no separators; lengths[i]
 * bases each), mean_coverage[i] the mean count of unitig i's k-mers and
 * kmers_count[i] their number.  With every output pointer null, *n_inout
 * and *seq_bytes_inout receive the unitig count and the total bases; with
 * outputs, they give the capacities (checked) and receive the sizes.  Any
 * output pointer may be null.  Built on the device on the first call and
 * cached in the result. */
int spk_result_unitigs(spk_result* res, int k_index, char* seqs, uint64_t* seq_bytes_inout,
                       uint64_t* lengths, double* mean_coverage, uint64_t* kmers_count,
                       uint64_t* n_inout);

int spk_result_free(spk_result* res);

/* ---- batched and serving entry points ---------------------------------- */
/* One counting job: a read set and its k values.  Host buffers must stay
 * valid until the job completes (spk_wait returns or spk_poll reports done). */
typedef struct spk_job {
  const uint8_t* data;
  size_t data_len;
  const uint64_t* offsets;
  const uint32_t* lengths;
  size_t n_reads;
  const uint32_t* ks;
  int n_k;
  spk_count_opts opts;
} spk_job;

/* Counts several independent read sets as one pipeline (samples of uneven
 * size, each with its own Bloom and table): one host thread uploads the jobs'
 * reads ahead on an upload stream while three lanes count them in order, so a
 * job's copies overlap the counts before it.  results[i] receives job i's
 * result, identical to spk_count on that job alone; if a job fails, every
 * result is freed and its status is returned.  Replaces the serial per-sample
 * (and per-k) loop of run_multik_assembly (src/multik.rs:109-178) for
 * independent samples. */
int spk_count_batch(spk_ctx* ctx, const spk_job* jobs, int n_jobs, spk_result** results);

/* The same pipeline with the results handed out as they finish.
 * spk_batch_start starts it (host buffers and the jobs array's contents must
 * stay valid until spk_batch_end; the ks arrays are copied).  spk_batch_next
 * waits for the next job in job order and hands over its result (the caller
 * frees it with spk_result_free), so the caller's downloads of one result
 * overlap the counts of the jobs after it; a failed job returns its status
 * with *index set and no result, and the batch goes on.  After the last job
 * it returns SPK_E_NOT_FOUND.  spk_batch_end waits for the batch's threads
 * and frees the results never handed out.  One batch runs at a time on a
 * context (a second spk_batch_start waits).  A batch result's later work
 * (downloads, unitigs) runs on the batch's result stream, in call order. */
typedef struct spk_batch spk_batch;
int spk_batch_start(spk_ctx* ctx, const spk_job* jobs, int n_jobs, spk_batch** batch);
int spk_batch_next(spk_batch* batch, int* index, spk_result** result);
int spk_batch_end(spk_batch* batch);

/* Serving loop.  spk_serve_start starts a scheduler thread that admits
 * submitted jobs in arrival order while at most max_inflight run, each on its
 * own stream: jobs run side by side while their estimated HBM needs together
 * stay within a sixteenth of hbm_budget_bytes (0 = 90% of the device memory
 * free at start), a job that needs more runs alone, and a job that needs more
 * than the whole budget is refused (SPK_E_ADMISSION). */
int spk_serve_start(spk_ctx* ctx, uint64_t hbm_budget_bytes, int max_inflight);
int spk_serve_stop(spk_ctx* ctx);
/* Estimated device bytes a job needs (Bloom + table + reads + outputs). */
int spk_job_hbm_estimate(const spk_job* job, uint64_t* bytes);
int spk_submit(spk_ctx* ctx, const spk_job* job, uint64_t* ticket);
/* *done = 1 when the job finished (successfully or not). */
int spk_poll(spk_ctx* ctx, uint64_t ticket, int* done);
/* Waits up to timeout_ms (<0: forever) and hands over the result.  Returns
 * the job's own status if it failed.  latency_ms (nullable) = submit->done. */
int spk_wait(spk_ctx* ctx, uint64_t ticket, int timeout_ms, spk_result** out, double* latency_ms);

/* ---- diagnostics --------------------------------------------------------- */
/* The count table's bounded wait for keys of k = 65..127.  The reference's
 * table is a mutex-guarded HashMap (src/assemble.rs:166-242) whose waits have
 * no bound; here a writer claims a slot, publishes its key and marks the slot
 * ready, and a reader that finds a slot claimed waits a bounded time for it.
 * This call counts one k-mer into a small table whose home slot for that
 * k-mer was left claimed and never published (what a writer gone mid-claim
 * would leave): the wait runs out after a fraction of a second and the call
 * returns SPK_E_TIMEOUT, with the context still usable.  No counterpart in the
 * reference. */
int spk_diag_stuck_claim(spk_ctx* ctx, uint32_t k);

#ifdef __cplusplus
}
#endif
#endif /* SPK_H */
