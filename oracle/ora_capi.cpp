// ora_capi.cpp -- C entry points of the CPU oracle for the Python test suite
// (ctypes).  TEST INFRASTRUCTURE ONLY: loaded by tests/, the smoke check and
// the CPU-baseline leg of bench.py; never by the product library.
//
// k-mer keys cross this boundary as little-endian u64 limbs of the reference
// Kmer256 (dna.rs:138): limb 0 = lo bits 0..63, limb 1 = lo bits 64..127,
// limb 2 = hi bits 0..63, limb 3 = hi bits 64..127.  A k-mer list uses
// ceil(k/32) limbs per key.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <map>

#include "spk_oracle.h"

using namespace ora;

static inline unsigned nlimbs(unsigned k) { return (k + 31) / 32; }
static inline Kmer256 from_limbs(const uint64_t* l, unsigned n) {
  uint64_t w[4] = {0, 0, 0, 0};
  for (unsigned i = 0; i < n && i < 4; i++) w[i] = l[i];
  Kmer256 x;
  x.lo = ((u128)w[1] << 64) | w[0];
  x.hi = ((u128)w[3] << 64) | w[2];
  return x;
}
static inline void to_limbs(const Kmer256& x, uint64_t* l, unsigned n) {
  uint64_t w[4] = {(uint64_t)x.lo, (uint64_t)(x.lo >> 64), (uint64_t)x.hi, (uint64_t)(x.hi >> 64)};
  for (unsigned i = 0; i < n && i < 4; i++) l[i] = w[i];
}

extern "C" {

// ---- dna.rs ---------------------------------------------------------------
int ora_base_to_2bit(uint8_t b) { return base_to_2bit(b); }
uint64_t ora_revcomp_u64(uint64_t x, unsigned k) { return revcomp_kmer_u64(x, k); }
uint64_t ora_canonical_u64(uint64_t x, unsigned k, int* is_rc) {
  bool r = false;
  uint64_t c = canonical_kmer_u64(x, k, &r);
  if (is_rc) *is_rc = r;
  return c;
}
int ora_string_to_kmer(const uint8_t* s, size_t len, unsigned k, uint64_t* out) {
  return string_to_kmer(s, len, k, out) ? 1 : 0;
}
int ora_k256_from_bytes(const uint8_t* s, size_t len, unsigned k, uint64_t* out4) {
  Kmer256 x;
  if (!k256_from_bytes(s, len, k, &x)) return 0;
  to_limbs(x, out4, 4);
  return 1;
}
void ora_k256_to_string(const uint64_t* in4, unsigned k, char* out) {
  std::string s = k256_to_string(from_limbs(in4, 4), k);
  memcpy(out, s.data(), s.size());
}
void ora_k256_revcomp(const uint64_t* in4, unsigned k, uint64_t* out4) {
  to_limbs(k256_revcomp(from_limbs(in4, 4), k), out4, 4);
}
int ora_k256_canonical(const uint64_t* in4, unsigned k, uint64_t* out4) {
  bool r = false;
  to_limbs(k256_canonical(from_limbs(in4, 4), k, &r), out4, 4);
  return r ? 1 : 0;
}
void ora_k256_extend_right(const uint64_t* in4, uint8_t b, unsigned k, uint64_t* out4) {
  to_limbs(k256_extend_right(from_limbs(in4, 4), b, k), out4, 4);
}
void ora_k256_prepend_left(const uint64_t* in4, uint8_t a, unsigned k, uint64_t* out4) {
  to_limbs(k256_prepend_left(from_limbs(in4, 4), a, k), out4, 4);
}

// ---- bloom.rs -------------------------------------------------------------
uint64_t ora_hash_kmer256(const uint64_t* in4, uint64_t seed) {
  return hash_kmer256(from_limbs(in4, 4), seed);
}
void ora_hash_batch(const uint64_t* keys4, size_t n, uint64_t seed, uint64_t* out) {
  for (size_t i = 0; i < n; i++) out[i] = hash_kmer256(from_limbs(keys4 + 4 * i, 4), seed);
}
void* ora_bloom_new(uint64_t capacity_bits) { return new TwoTierFilter(capacity_bits); }
void ora_bloom_free(void* f) { delete (TwoTierFilter*)f; }
uint64_t ora_bloom_size_bits(void* f) { return ((TwoTierFilter*)f)->size_bits; }
uint64_t ora_bloom_num_words(void* f) { return ((TwoTierFilter*)f)->num_words; }
uint64_t ora_bloom_memory_usage_bytes(void* f) { return ((TwoTierFilter*)f)->memory_usage_bytes(); }
int ora_bloom_insert_k256(void* f, const uint64_t* in4) {
  return ((TwoTierFilter*)f)->insert_kmer256(from_limbs(in4, 4)) ? 1 : 0;
}
int ora_bloom_is_solid_k256(void* f, const uint64_t* in4) {
  return ((TwoTierFilter*)f)->is_solid_kmer256(from_limbs(in4, 4)) ? 1 : 0;
}
int ora_bloom_insert_u64(void* f, uint64_t x) { return ((TwoTierFilter*)f)->insert(x) ? 1 : 0; }
int ora_bloom_is_solid_u64(void* f, uint64_t x) { return ((TwoTierFilter*)f)->is_solid(x) ? 1 : 0; }
void ora_bloom_download(void* f, uint64_t* seen, uint64_t* solid) {
  TwoTierFilter* t = (TwoTierFilter*)f;
  if (seen) memcpy(seen, t->seen.data(), t->num_words * 8);
  if (solid) memcpy(solid, t->solid.data(), t->num_words * 8);
}

// ---- packed_reads.rs ------------------------------------------------------
void* ora_packed_new() { return new PackedReads(); }
void ora_packed_free(void* p) { delete (PackedReads*)p; }
void ora_packed_pack_clean(void* p, const uint8_t* s, size_t len) { ((PackedReads*)p)->pack_clean(s, len); }
void ora_packed_ingest_read(void* p, const uint8_t* s, size_t len) { ((PackedReads*)p)->ingest_read(s, len); }
// Reads are passed as one concatenated buffer plus per-read lengths.
void* ora_packed_from_paired(const char* r1, const uint64_t* l1, size_t n1, const char* r2,
                             const uint64_t* l2, size_t n2) {
  std::vector<std::string> a, b;
  size_t o = 0;
  for (size_t i = 0; i < n1; i++) { a.emplace_back(r1 + o, l1[i]); o += l1[i]; }
  o = 0;
  for (size_t i = 0; i < n2; i++) { b.emplace_back(r2 + o, l2[i]); o += l2[i]; }
  return new PackedReads(from_paired_slices(a, b));
}
void ora_packed_sizes(void* p, uint64_t* n_reads, uint64_t* data_len, uint64_t* pe_count,
                      uint64_t* n_sidecar) {
  PackedReads* r = (PackedReads*)p;
  *n_reads = r->size();
  *data_len = r->data.size();
  *pe_count = r->pe_count;
  *n_sidecar = r->ambiguous_sidecar.size();
}
void ora_packed_copy(void* p, uint8_t* data, uint64_t* offsets, uint32_t* lengths) {
  PackedReads* r = (PackedReads*)p;
  if (data) memcpy(data, r->data.data(), r->data.size());
  if (offsets) memcpy(offsets, r->offsets.data(), r->offsets.size() * 8);
  if (lengths) memcpy(lengths, r->lengths.data(), r->lengths.size() * 4);
}
// FASTQ / FASTA texts (decompressed) ingested as from_paired_files (t2 != null)
// or append_from_file on an empty store; null on a malformed text (*err_out
// gets the message, up to 255 bytes).
void* ora_packed_from_texts(const uint8_t* t1, size_t l1, const uint8_t* t2, size_t l2, char* err_out) {
  PackedReads* r = new PackedReads();
  std::string err;
  const bool ok = t2 ? from_paired_texts(t1, l1, t2, l2, r, &err) : from_single_text(t1, l1, r, &err);
  if (!ok) {
    delete r;
    if (err_out) snprintf(err_out, 256, "%s", err.c_str());
    return nullptr;
  }
  return r;
}
size_t ora_packed_sidecar_get(void* p, size_t i, uint8_t* out) {
  const std::string& s = ((PackedReads*)p)->ambiguous_sidecar[i];
  if (out) memcpy(out, s.data(), s.size());
  return s.size();
}
size_t ora_packed_get_read(void* p, size_t idx, uint8_t* out) {
  std::vector<uint8_t> buf;
  ((PackedReads*)p)->get_read(idx, buf);
  if (out) memcpy(out, buf.data(), buf.size());
  return buf.size();
}

// ---- assemble.rs Stages 2-3 -------------------------------------------------
// threads == 0 selects the serial restatement; threads >= 1 the threaded one.
void* ora_count(const uint8_t* data, size_t data_len, const uint64_t* offsets,
                const uint32_t* lengths, size_t n_reads, unsigned k, uint64_t bloom_bits,
                int mode, int threads, int keep_bloom) {
  PackedReads pr;
  pr.data.assign(data, data + data_len);
  pr.offsets.assign(offsets, offsets + n_reads);
  pr.lengths.assign(lengths, lengths + n_reads);
  CountResult* r = new CountResult();
  if (threads <= 0) {
    // mode bit 8: the error-correcting Stage 3 (assemble.rs:183-191)
    count_serial(pr, k, bloom_bits, (Mode)(mode & 0xFF), r, (mode & 0x100) != 0);
    if (!keep_bloom) { r->seen.clear(); r->solid.clear(); }
  } else {
    count_threaded(pr, k, bloom_bits, threads, (Mode)(mode & 0xFF), keep_bloom != 0, r, (mode & 0x100) != 0);
  }
  return r;
}
void ora_count_free(void* r) { delete (CountResult*)r; }
// The threaded count with Stage 3 restricted to the first stage3_reads reads
// (Stage 2 over all of them): a bounded sample of a full-size job's Stage 3.
void* ora_count_sample3(const uint8_t* data, size_t data_len, const uint64_t* offsets, const uint32_t* lengths,
                        size_t n_reads, unsigned k, uint64_t bloom_bits, int mode, int threads, size_t stage3_reads) {
  PackedReads pr;
  pr.data.assign(data, data + data_len);
  pr.offsets.assign(offsets, offsets + n_reads);
  pr.lengths.assign(lengths, lengths + n_reads);
  CountResult* r = new CountResult();
  count_threaded(pr, k, bloom_bits, threads, (Mode)(mode & 0xFF), false, r, (mode & 0x100) != 0, stage3_reads);
  return r;
}
// Unitigs of a sorted solid list (keys as ceil(k/32) limbs): returns a handle.
void* ora_unitigs(const uint64_t* keys, const uint32_t* counts, size_t n, unsigned k) {
  const unsigned L = nlimbs(k);
  std::vector<Kmer256> s(n);
  for (size_t i = 0; i < n; i++) s[i] = from_limbs(keys + i * L, L);
  std::vector<uint32_t> c(counts, counts + n);
  return new std::vector<Unitig>(unitigs(s, c, k));
}
size_t ora_unitigs_count(void* h) { return ((std::vector<Unitig>*)h)->size(); }
size_t ora_unitigs_bases(void* h) {
  size_t b = 0;
  for (auto& u : *(std::vector<Unitig>*)h) b += u.sequence.size();
  return b;
}
void ora_unitigs_get(void* h, char* seqs, uint64_t* lengths, double* cov, uint64_t* kmers) {
  size_t o = 0, i = 0;
  for (auto& u : *(std::vector<Unitig>*)h) {
    memcpy(seqs + o, u.sequence.data(), u.sequence.size());
    o += u.sequence.size();
    lengths[i] = u.sequence.size();
    cov[i] = u.mean_coverage;
    kmers[i] = u.kmers_count;
    i++;
  }
}
void ora_unitigs_free(void* h) { delete (std::vector<Unitig>*)h; }
// Overwrites the filter's tiers (num_words words each; either may be null).
void ora_bloom_load(void* f, const uint64_t* seen, const uint64_t* solid) {
  auto* b = (TwoTierFilter*)f;
  if (seen) memcpy(b->seen.data(), seen, b->num_words * 8);
  if (solid) memcpy(b->solid.data(), solid, b->num_words * 8);
}
// ErrorCorrector::correct_read_in_place on one ASCII read, in place.
int ora_correct_ascii(void* f, unsigned k, uint8_t* seq, size_t len) {
  std::vector<uint8_t> v(seq, seq + len);
  const bool m = correct_read_in_place(k, v, *(TwoTierFilter*)f);
  memcpy(seq, v.data(), len);
  return m ? 1 : 0;
}
// The Stage 3 use (src/assemble.rs:183-191): every packed read decoded,
// corrected and its changed bases written back into a copy of the packed data
// (out_data, data_len bytes); corrected[i] = 1 if read i changed.  Returns the
// number of corrected reads.
size_t ora_correct_packed(void* f, unsigned k, const uint8_t* data, size_t data_len, const uint64_t* offs,
                          const uint32_t* lens, size_t n, uint8_t* out_data, uint8_t* corrected) {
  memcpy(out_data, data, data_len);
  size_t nc = 0;
  std::vector<uint8_t> buf;
  for (size_t r = 0; r < n; r++) {
    const uint32_t L = lens[r];
    buf.resize(L);
    for (uint32_t j = 0; j < L; j++)
      buf[j] = "ACGT"[(data[offs[r] + j / 4] >> (6 - 2 * (j % 4))) & 3];
    const std::vector<uint8_t> before(buf);
    const bool m = L >= k && correct_read_in_place(k, buf, *(TwoTierFilter*)f);
    corrected[r] = m ? 1 : 0;
    nc += m;
    for (uint32_t j = 0; j < L; j++) {
      if (buf[j] == before[j]) continue;
      uint8_t& byte = out_data[offs[r] + j / 4];
      const unsigned sh = 6 - 2 * (j % 4);
      byte = (uint8_t)((byte & ~(3u << sh)) | ((unsigned)base_to_2bit(buf[j]) << sh));
    }
  }
  return nc;
}
// prior contigs (ASCII) concatenated in seqs, contig i = seqs[offs[i] .. offs[i] + lens[i])
void ora_count_inject_priors(void* r, const uint8_t* seqs, const uint64_t* offs, const uint32_t* lens,
                             size_t n, unsigned k, uint32_t boost) {
  std::vector<std::vector<uint8_t>> pr(n);
  for (size_t i = 0; i < n; i++) pr[i].assign(seqs + offs[i], seqs + offs[i] + lens[i]);
  inject_priors((CountResult*)r, pr, k, boost);
}
size_t ora_count_size(void* r, uint32_t min_count) {
  size_t n = 0;
  for (auto& e : ((CountResult*)r)->table) n += e.count >= min_count;
  return n;
}
size_t ora_count_table(void* r, unsigned k, uint32_t min_count, uint64_t* keys, uint32_t* counts) {
  unsigned L = nlimbs(k);
  size_t n = 0;
  for (auto& e : ((CountResult*)r)->table) {
    if (e.count < min_count) continue;
    if (keys) to_limbs(e.key, keys + n * L, L);
    if (counts) counts[n] = e.count;
    n++;
  }
  return n;
}
size_t ora_count_bloom_words(void* r) { return ((CountResult*)r)->seen.size(); }
void ora_count_bloom(void* r, uint64_t* seen, uint64_t* solid) {
  CountResult* c = (CountResult*)r;
  if (seen) memcpy(seen, c->seen.data(), c->seen.size() * 8);
  if (solid) memcpy(solid, c->solid.data(), c->solid.size() * 8);
}
// out: occurrences, admitted_occurrences, stage2 s, stage3 s, total s, corrected reads
void ora_count_stats(void* r, double* out) {
  CountResult* c = (CountResult*)r;
  out[0] = (double)c->occurrences;
  out[1] = (double)c->admitted_occurrences;
  out[2] = c->seconds_stage2;
  out[3] = c->seconds_stage3;
  out[4] = c->seconds_total;
  out[5] = (double)c->corrected_reads;
}

uint32_t ora_cutoff(const uint32_t* counts, size_t n, double min_coverage) {
  std::vector<uint32_t> v(counts, counts + n);
  return determine_solid_kmer_cutoff(v, min_coverage);
}

// Edge list for a sorted solid set.  Returns the number of edges; the caller
// frees *out with ora_free.  Edge keys use ceil((k+1)/32) limbs.
size_t ora_edges(const uint64_t* solid_keys, size_t n, unsigned k, uint64_t** out) {
  unsigned L = nlimbs(k), Le = nlimbs(k + 1);
  std::vector<Kmer256> s(n);
  for (size_t i = 0; i < n; i++) s[i] = from_limbs(solid_keys + i * L, L);
  std::sort(s.begin(), s.end());
  std::vector<Kmer256> e = edges(s, k);
  uint64_t* o = (uint64_t*)malloc(std::max<size_t>(e.size(), 1) * Le * 8);
  for (size_t i = 0; i < e.size(); i++) to_limbs(e[i], o + i * Le, Le);
  *out = o;
  return e.size();
}
void ora_free(void* p) { free(p); }

// ---- one rank's share of the sharded design (several GPUs) ----------------
// Rank r of G owns the Bloom words [r W / G, (r + 1) W / G) and the k-mers
// whose hash_kmer256(seed 1) falls in the r-th of G equal ranges of 2^64.
// Phase 1: the rank applies the twice-tier inserts (bloom.rs:95-97 with the
// twice tier) of every k-mer occurrence whose position lies in its words;
// the tiers are order-free, so the ranks' word ranges side by side are the
// single filter.  Phase 2, with the gathered twice tier: the rank counts
// every occurrence of its own k-mers (assemble.rs:175-219 without the gate)
// and admits a k-mer seen once when its three twice bits are set.  The
// ranks' tables are disjoint; merged and sorted they are the single table.
// Test infrastructure: the restatement the multi-rank tests check the
// partition and the exchange against.
static uint32_t owner_of(const Kmer256& c, unsigned world) {
  return (uint32_t)(((unsigned __int128)hash_kmer256(c, SEED1) * world) >> 64);
}
void ora_shard_bloom(const uint8_t* data, size_t data_len, const uint64_t* offsets, const uint32_t* lengths,
                     size_t n_reads, unsigned k, uint64_t bloom_bits, uint64_t word_lo, uint64_t word_hi,
                     uint64_t* seen, uint64_t* twice) {
  PackedReads pr;
  pr.data.assign(data, data + data_len);
  pr.offsets.assign(offsets, offsets + n_reads);
  pr.lengths.assign(lengths, lengths + n_reads);
  uint64_t num_words = std::max<uint64_t>((bloom_bits + 63) / 64, 1), size_bits = num_words * 64;
  memset(seen, 0, (word_hi - word_lo) * 8);
  memset(twice, 0, (word_hi - word_lo) * 8);
  std::vector<uint8_t> buf;
  for (size_t idx = 0; idx < pr.size(); idx++) {
    pr.get_read(idx, buf);
    for (size_t i = 0; i + k <= buf.size(); i++) {
      Kmer256 km;
      if (!k256_from_bytes(buf.data() + i, k, k, &km)) continue;
      const Kmer256 can = k256_canonical(km, k, nullptr);
      const uint64_t h[3] = {hash_kmer256(can, SEED1) % size_bits, hash_kmer256(can, SEED2) % size_bits,
                             hash_kmer256(can, SEED3) % size_bits};
      for (int j = 0; j < 3; j++) {
        const uint64_t w = h[j] / 64, b = 1ULL << (h[j] % 64);
        if (w < word_lo || w >= word_hi) continue;
        if (seen[w - word_lo] & b) twice[w - word_lo] |= b;
        seen[w - word_lo] |= b;
      }
    }
  }
}
void* ora_shard_count(const uint8_t* data, size_t data_len, const uint64_t* offsets, const uint32_t* lengths,
                      size_t n_reads, unsigned k, uint64_t bloom_bits, const uint64_t* twice, unsigned rank,
                      unsigned world) {
  PackedReads pr;
  pr.data.assign(data, data + data_len);
  pr.offsets.assign(offsets, offsets + n_reads);
  pr.lengths.assign(lengths, lengths + n_reads);
  uint64_t num_words = std::max<uint64_t>((bloom_bits + 63) / 64, 1), size_bits = num_words * 64;
  std::map<Kmer256, uint32_t> cnt;
  std::vector<uint8_t> buf;
  for (size_t idx = 0; idx < pr.size(); idx++) {
    pr.get_read(idx, buf);
    for (size_t i = 0; i + k <= buf.size(); i++) {
      Kmer256 km;
      if (!k256_from_bytes(buf.data() + i, k, k, &km)) continue;
      const Kmer256 can = k256_canonical(km, k, nullptr);
      if (owner_of(can, world) == rank) cnt[can]++;
    }
  }
  CountResult* r = new CountResult();
  for (auto& kv : cnt) {
    bool admit = kv.second >= 2;
    if (!admit) {
      admit = true;
      for (uint64_t seed : {SEED1, SEED2, SEED3}) {
        const uint64_t h = hash_kmer256(kv.first, seed) % size_bits;
        admit = admit && ((twice[h / 64] >> (h % 64)) & 1);
      }
    }
    if (admit) r->table.push_back(CountEntry{kv.first, kv.second});
  }
  return r;  // sorted: std::map order is Kmer256 order
}

}  // extern "C"
