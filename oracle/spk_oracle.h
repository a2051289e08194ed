// spk_oracle.h -- CPU restatement of the spades-rs k-mer counting path.
//
// TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA library is
// compared against, and the timed CPU baseline ("C++ restatement of spades-rs
// Stages 2-3").  It is never linked into, loaded by, or called from the
// product library (libspk).  Only tests/, the smoke check and the
// cpu-baseline leg of bench.py load it.
//
// Every function cites the reference file:line it restates (paths are
// relative to the spades-rs project root).  The reference is Rust and cannot
// be built on this machine, so this file is a line-by-line restatement of the
// algorithm, not a binding.
#pragma once
#include <cstddef>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>

namespace ora {

typedef unsigned __int128 u128;

// src/dna.rs:138  `pub struct Kmer256(pub u128, pub u128)`; derived Ord is
// lexicographic on (lo, hi).
struct Kmer256 {
  u128 lo = 0, hi = 0;
  bool operator==(const Kmer256& o) const { return lo == o.lo && hi == o.hi; }
  bool operator!=(const Kmer256& o) const { return !(*this == o); }
  bool operator<(const Kmer256& o) const { return lo < o.lo || (lo == o.lo && hi < o.hi); }
  bool operator<=(const Kmer256& o) const { return !(o < *this); }
};

// ---- src/dna.rs ----------------------------------------------------------
extern const uint8_t ASCII_TO_2BIT[256];                       // dna.rs:11-22
int base_to_2bit(uint8_t b);                                    // dna.rs:30-37 (-1 == None)
uint8_t bit2_to_base(uint8_t v);                                // dna.rs:41-43
uint64_t revcomp_kmer_u64(uint64_t kmer, unsigned k);           // dna.rs:65-78
uint64_t canonical_kmer_u64(uint64_t kmer, unsigned k, bool* is_rc);  // dna.rs:82-89
bool string_to_kmer(const uint8_t* s, size_t len, unsigned k, uint64_t* out);  // dna.rs:104-114
std::string kmer_to_string(uint64_t kmer, unsigned k);          // dna.rs:92-100
u128 revcomp_kmer_u128(u128 kmer, unsigned k);                  // dna.rs:118-132
Kmer256 k256_revcomp(const Kmer256& x, unsigned k);             // dna.rs:152-180
Kmer256 k256_canonical(const Kmer256& x, unsigned k, bool* is_rc);  // dna.rs:185-192
Kmer256 k256_extend_right(const Kmer256& x, uint8_t b, unsigned k); // dna.rs:196-221
Kmer256 k256_prepend_left(const Kmer256& x, uint8_t a, unsigned k); // dna.rs:225-245
uint8_t k256_last_base(const Kmer256& x, unsigned k);           // dna.rs:249-258
uint8_t k256_first_base(const Kmer256& x, unsigned k);          // dna.rs:262-271
std::string k256_to_string(const Kmer256& x, unsigned k);       // dna.rs:274-295
bool k256_from_bytes(const uint8_t* s, size_t len, unsigned k, Kmer256* out);  // dna.rs:299-321

// ---- src/bloom.rs --------------------------------------------------------
static const uint64_t SEED1 = 0x517cc1b727220a95ULL;  // bloom.rs:84
static const uint64_t SEED2 = 0x9e3779b97f4a7c15ULL;  // bloom.rs:85
static const uint64_t SEED3 = 0x6c62272e07bb0142ULL;  // bloom.rs:86
uint64_t hash_kmer256(const Kmer256& k, uint64_t seed);          // bloom.rs:61-78

// Admission semantics of the count table.
//  REF   : reference TwoTierFilter (bloom.rs:83-126).  A k-mer is promoted to
//          the solid tier when all three seen bits were already set when it was
//          inserted, so the solid tier depends on insertion order.
//  TWICE : order-free "twice-hit" tier used by the GPU.  Each seen fetch_or
//          that finds its bit already set also sets the same bit in the twice
//          tier; a k-mer is admitted when all three twice bits are set.  Its
//          final state does not depend on insertion order, and every k-mer that
//          occurs at least twice is admitted.
enum Mode { MODE_REF = 0, MODE_TWICE = 1 };

// bloom.rs:13-131.  Plain (non-atomic) words for the serial oracle; the
// threaded CPU baseline uses its own atomic copy.
struct TwoTierFilter {
  uint64_t size_bits = 0, num_words = 0;
  std::vector<uint64_t> seen, solid;  // `solid` holds the twice tier in MODE_TWICE
  explicit TwoTierFilter(uint64_t capacity_bits);               // bloom.rs:26-43
  bool insert_kmer256(const Kmer256& k);                        // bloom.rs:83-107
  bool insert_twice(const Kmer256& k);                          // twice-tier insert
  bool is_solid_kmer256(const Kmer256& k) const;                // bloom.rs:111-126
  bool insert(uint64_t k) { Kmer256 x; x.lo = k; return insert_kmer256(x); }  // bloom.rs:48-50
  bool is_solid(uint64_t k) const { Kmer256 x; x.lo = k; return is_solid_kmer256(x); }  // bloom.rs:54-56
  uint64_t memory_usage_bytes() const { return num_words * 8 * 2; }  // bloom.rs:129-131
};

// ---- src/packed_reads.rs -------------------------------------------------
struct PackedReads {
  std::vector<uint8_t> data;       // packed_reads.rs:44
  std::vector<uint64_t> offsets;   // packed_reads.rs:46
  std::vector<uint32_t> lengths;   // packed_reads.rs:48
  uint64_t pe_count = 0;           // packed_reads.rs:53
  std::vector<std::string> ambiguous_sidecar;  // packed_reads.rs:58
  size_t size() const { return lengths.size(); }
  void pack_clean(const uint8_t* read, size_t len);             // packed_reads.rs:547-578
  void get_read(size_t idx, std::vector<uint8_t>& buf) const;   // packed_reads.rs:592-613
  void ingest_read(const uint8_t* read, size_t len);            // packed_reads.rs:513-517
  void ingest_trimmed_unpaired(const uint8_t* t, size_t len);   // packed_reads.rs:521-540
  void append_packed(const PackedReads& o);                     // packed_reads.rs:291-298
};
// packed_reads.rs:438-461 + 481-489 + 668-690
PackedReads from_paired_slices(const std::vector<std::string>& r1,
                               const std::vector<std::string>& r2);
// FastxReader::open + next_seq (packed_reads.rs:69-234) over an in-memory
// (decompressed) FASTQ or FASTA text: the sequence of every record, in order.
// false with *err set for a malformed text.
bool fastx_records(const uint8_t* text, size_t len, std::vector<std::string>* out, std::string* err);
// from_paired_files (packed_reads.rs:324-381) and append_from_file on an
// empty store (packed_reads.rs:493-504) over in-memory texts.
bool from_paired_texts(const uint8_t* t1, size_t l1, const uint8_t* t2, size_t l2, PackedReads* out,
                       std::string* err);
bool from_single_text(const uint8_t* t, size_t l, PackedReads* out, std::string* err);

// ---- src/assemble.rs Stages 2-3 -------------------------------------------
struct CountEntry { Kmer256 key; uint32_t count; };

struct CountResult {
  std::vector<CountEntry> table;    // every admitted k-mer, sorted by key
  std::vector<uint64_t> seen;       // Bloom seen tier (bloom.rs:19)
  std::vector<uint64_t> solid;      // solid tier (REF) or twice tier (TWICE)
  uint64_t occurrences = 0;         // k-mer positions visited per pass
  uint64_t admitted_occurrences = 0;
  uint64_t corrected_reads = 0;     // reads the Stage 3 error correction changed
  double seconds_stage2 = 0, seconds_stage3 = 0, seconds_total = 0;
};

// Serial restatement of assemble.rs:129-242: reads in index order, positions
// left to right.  correct: the config.error_correct branch (:183-191), every
// read corrected against the filter before its k-mers are counted.
void count_serial(const PackedReads& pr, unsigned k, uint64_t bloom_bits, Mode mode,
                  CountResult* out, bool correct = false);
// Threaded restatement used as the CPU baseline: same chunking
// (assemble.rs:137-139), sharded maps behind mutexes with 256-entry local
// buffers (assemble.rs:167-218), shard merge (assemble.rs:238-242).
void count_threaded(const PackedReads& pr, unsigned k, uint64_t bloom_bits, int threads,
                    Mode mode, bool keep_bloom, CountResult* out, bool correct = false,
                    size_t stage3_reads = SIZE_MAX);

// assemble.rs:692-735
uint32_t determine_solid_kmer_cutoff(const std::vector<uint32_t>& counts, double min_coverage);

// src/assemble.rs:267-283: every k-window of every prior contig that
// Kmer256::from_bytes accepts adds `boost` to its canonical k-mer's count,
// inserting the k-mer when the table does not hold it.  The table stays
// sorted by key.
void inject_priors(CountResult* r, const std::vector<std::vector<uint8_t>>& priors, unsigned k,
                   uint32_t boost);

// CompactedGraph::build (src/graph.rs:65-235): maximal non-branching paths
// of the solid k-mers.  The reference walks a HashSet, whose order (and so
// each unitig's orientation, its position in the output and where an
// isolated cycle is cut) depends on the hasher; here the solid k-mers are
// walked in sorted order.  Each unitig is then put in the orientation that
// is not greater than its reverse complement and the list is sorted by
// sequence, which is the same for every walk order except the cut of a
// cycle (taken at the cycle's smallest k-mer, as the sorted walk does).
struct Unitig {
  std::string sequence;
  double mean_coverage;
  size_t kmers_count;
};
std::vector<Unitig> unitigs(const std::vector<Kmer256>& solid_sorted,
                            const std::vector<uint32_t>& counts, unsigned k);

// graph.rs:78-102: the (k+1)-mer edge set implied by get_successors over the
// solid set, as canonical (k+1)-mers, sorted.
std::vector<Kmer256> edges(const std::vector<Kmer256>& solid_sorted, unsigned k);

// hammer.rs:34-121: ErrorCorrector::correct_read_in_place, single-base
// substitutions against the filter's solid tier; true if a base changed.
bool correct_read_in_place(unsigned k, std::vector<uint8_t>& seq, const TwoTierFilter& filter);

}  // namespace ora
