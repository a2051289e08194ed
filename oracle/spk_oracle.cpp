// spk_oracle.cpp -- CPU restatement of the spades-rs k-mer counting path.
// TEST INFRASTRUCTURE ONLY (see spk_oracle.h): the checker and the timed CPU
// baseline; never part of the product library.
#include "spk_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>

namespace ora {

// ---------------------------------------------------------------------------
// src/dna.rs
// ---------------------------------------------------------------------------
// dna.rs:11-22
const uint8_t ASCII_TO_2BIT[256] = {
#define X 0xFF
    X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X, X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,
    X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X, X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,
    X,0,X,1,X,X,X,2,X,X,X,X,X,X,X,X, X,X,X,X,3,X,X,X,X,X,X,X,X,X,X,X,
    X,0,X,1,X,X,X,2,X,X,X,X,X,X,X,X, X,X,X,X,3,X,X,X,X,X,X,X,X,X,X,X,
    X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X, X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,
    X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X, X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,
    X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X, X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,
    X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X, X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,X,
#undef X
};

// dna.rs:30-37
int base_to_2bit(uint8_t b) {
  uint8_t v = ASCII_TO_2BIT[b];
  return v != 0xFF ? int(v) : -1;
}
// dna.rs:41-43
uint8_t bit2_to_base(uint8_t v) { return "ACGT"[v & 3]; }

static uint64_t reverse_bits64(uint64_t x) {
  x = ((x >> 1) & 0x5555555555555555ULL) | ((x & 0x5555555555555555ULL) << 1);
  x = ((x >> 2) & 0x3333333333333333ULL) | ((x & 0x3333333333333333ULL) << 2);
  x = ((x >> 4) & 0x0F0F0F0F0F0F0F0FULL) | ((x & 0x0F0F0F0F0F0F0F0FULL) << 4);
  return __builtin_bswap64(x);
}
static u128 reverse_bits128(u128 x) {
  uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
  return ((u128)reverse_bits64(lo) << 64) | (u128)reverse_bits64(hi);
}
static const u128 M55 = ((u128)0x5555555555555555ULL << 64) | (u128)0x5555555555555555ULL;

// dna.rs:65-78
uint64_t revcomp_kmer_u64(uint64_t kmer, unsigned k) {
  if (k == 0 || k > 32) return 0;
  kmer = reverse_bits64(~kmer);
  kmer = ((kmer >> 1) & 0x5555555555555555ULL) | ((kmer & 0x5555555555555555ULL) << 1);
  return kmer >> (2 * (32 - k));
}
// dna.rs:82-89
uint64_t canonical_kmer_u64(uint64_t kmer, unsigned k, bool* is_rc) {
  uint64_t rc = revcomp_kmer_u64(kmer, k);
  if (kmer <= rc) { if (is_rc) *is_rc = false; return kmer; }
  if (is_rc) *is_rc = true;
  return rc;
}
// dna.rs:104-114
bool string_to_kmer(const uint8_t* s, size_t len, unsigned k, uint64_t* out) {
  if (k == 0 || k > 32 || len < k) return false;
  uint64_t v = 0;
  for (unsigned i = 0; i < k; i++) {
    int c = base_to_2bit(s[i]);
    if (c < 0) return false;
    v = (v << 2) | (uint64_t)c;
  }
  *out = v;
  return true;
}
// dna.rs:92-100
std::string kmer_to_string(uint64_t kmer, unsigned k) {
  if (k > 32) k = 32;
  std::string s(k, 'A');
  for (int i = int(k) - 1; i >= 0; i--) { s[i] = bit2_to_base(kmer & 3); kmer >>= 2; }
  return s;
}
// dna.rs:118-132
u128 revcomp_kmer_u128(u128 kmer, unsigned k) {
  if (k == 0 || k > 64) return 0;
  kmer = reverse_bits128(~kmer);
  kmer = ((kmer >> 1) & M55) | ((kmer & M55) << 1);
  return k == 64 ? kmer : kmer >> (2 * (64 - k));
}
// dna.rs:152-180
Kmer256 k256_revcomp(const Kmer256& x, unsigned k) {
  Kmer256 r;
  if (k == 0 || k > 128) return r;
  if (k <= 64) { r.lo = revcomp_kmer_u128(x.lo, k); return r; }
  unsigned k2 = k - 64;
  u128 lo_rc = revcomp_kmer_u128(x.lo, 64);
  u128 hi_rc = revcomp_kmer_u128(x.hi, k2);
  unsigned shift_lo = 2 * (64 - k2);
  u128 a = shift_lo >= 128 ? (u128)0 : (hi_rc << shift_lo);
  u128 b = k2 >= 64 ? (u128)0 : (lo_rc >> (2 * k2));
  u128 mask_hi = k2 >= 64 ? ~(u128)0 : (((u128)1 << (2 * k2)) - 1);
  r.lo = a | b;
  r.hi = lo_rc & mask_hi;
  return r;
}
// dna.rs:185-192
Kmer256 k256_canonical(const Kmer256& x, unsigned k, bool* is_rc) {
  Kmer256 rc = k256_revcomp(x, k);
  if (x <= rc) { if (is_rc) *is_rc = false; return x; }
  if (is_rc) *is_rc = true;
  return rc;
}
// dna.rs:196-221
Kmer256 k256_extend_right(const Kmer256& x, uint8_t b, unsigned k) {
  Kmer256 r;
  if (k == 0 || k > 128) return r;
  u128 b2 = (u128)(b & 3);
  if (k <= 64) {
    u128 mask = k == 64 ? ~(u128)0 : (((u128)1 << (2 * k)) - 1);
    r.lo = ((x.lo << 2) | b2) & mask;
    return r;
  }
  unsigned k2 = k - 64;
  u128 mask_hi = k2 == 64 ? ~(u128)0 : (((u128)1 << (2 * k2)) - 1);
  u128 s64 = (x.hi >> (2 * (k2 - 1))) & 3;
  r.lo = (x.lo << 2) | s64;
  r.hi = ((x.hi << 2) | b2) & mask_hi;
  return r;
}
// dna.rs:225-245
Kmer256 k256_prepend_left(const Kmer256& x, uint8_t a, unsigned k) {
  Kmer256 r;
  if (k == 0 || k > 128) return r;
  u128 a2 = (u128)(a & 3);
  if (k <= 64) { r.lo = (x.lo >> 2) | (a2 << (2 * (k - 1))); return r; }
  unsigned k2 = k - 64;
  u128 mask_hi = k2 == 64 ? ~(u128)0 : (((u128)1 << (2 * k2)) - 1);
  u128 s63 = x.lo & 3;
  r.lo = (x.lo >> 2) | (a2 << 126);
  r.hi = ((x.hi >> 2) | (s63 << (2 * (k2 - 1)))) & mask_hi;
  return r;
}
// dna.rs:249-258
uint8_t k256_last_base(const Kmer256& x, unsigned k) {
  if (k == 0) return 0;
  return k <= 64 ? uint8_t(x.lo & 3) : uint8_t(x.hi & 3);
}
// dna.rs:262-271
uint8_t k256_first_base(const Kmer256& x, unsigned k) {
  if (k == 0) return 0;
  return k <= 64 ? uint8_t((x.lo >> (2 * (k - 1))) & 3) : uint8_t((x.lo >> 126) & 3);
}
// dna.rs:274-295
std::string k256_to_string(const Kmer256& x, unsigned k) {
  std::string s(k, 'A');
  if (k <= 64) {
    u128 v = x.lo;
    for (int i = int(k) - 1; i >= 0; i--) { s[i] = bit2_to_base(uint8_t(v & 3)); v >>= 2; }
  } else {
    u128 v = x.lo;
    for (int i = 63; i >= 0; i--) { s[i] = bit2_to_base(uint8_t(v & 3)); v >>= 2; }
    u128 h = x.hi;
    for (int i = int(k) - 1; i >= 64; i--) { s[i] = bit2_to_base(uint8_t(h & 3)); h >>= 2; }
  }
  return s;
}
// dna.rs:299-321
bool k256_from_bytes(const uint8_t* s, size_t len, unsigned k, Kmer256* out) {
  if (k == 0 || len < k || k > 128) return false;
  u128 lo = 0, hi = 0;
  if (k <= 64) {
    for (unsigned i = 0; i < k; i++) {
      int c = base_to_2bit(s[i]);
      if (c < 0) return false;
      lo = (lo << 2) | (u128)c;
    }
  } else {
    for (unsigned i = 0; i < 64; i++) {
      int c = base_to_2bit(s[i]);
      if (c < 0) return false;
      lo = (lo << 2) | (u128)c;
    }
    for (unsigned i = 64; i < k; i++) {
      int c = base_to_2bit(s[i]);
      if (c < 0) return false;
      hi = (hi << 2) | (u128)c;
    }
  }
  out->lo = lo;
  out->hi = hi;
  return true;
}

// ---------------------------------------------------------------------------
// src/bloom.rs
// ---------------------------------------------------------------------------
static inline uint64_t rotl64(uint64_t x, unsigned r) { return (x << r) | (x >> (64 - r)); }

// bloom.rs:61-78 (constants verbatim; all products wrap mod 2^64)
uint64_t hash_kmer256(const Kmer256& km, uint64_t seed) {
  uint64_t w0 = (uint64_t)km.lo;
  uint64_t w1 = (uint64_t)(km.lo >> 64);
  uint64_t w2 = (uint64_t)km.hi;
  uint64_t w3 = (uint64_t)(km.hi >> 64);
  uint64_t x = w0 ^ seed;
  x = (x ^ (rotl64(w1, 21) * 0x9e3779b97f4a7c15ULL)) * 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x = (x ^ (rotl64(w2, 43) * 0xbf58476d1ce4e5b9ULL)) * 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  x = (x ^ (rotl64(w3, 11) * 0x94d049bb133111ebULL)) * 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  return x;
}

// bloom.rs:26-43
TwoTierFilter::TwoTierFilter(uint64_t capacity_bits) {
  num_words = (capacity_bits + 63) / 64;
  if (num_words < 1) num_words = 1;
  size_bits = num_words * 64;
  seen.assign(num_words, 0);
  solid.assign(num_words, 0);
}

// bloom.rs:83-107
bool TwoTierFilter::insert_kmer256(const Kmer256& km) {
  uint64_t h1 = hash_kmer256(km, SEED1) % size_bits;
  uint64_t h2 = hash_kmer256(km, SEED2) % size_bits;
  uint64_t h3 = hash_kmer256(km, SEED3) % size_bits;
  uint64_t w1 = h1 / 64, b1 = 1ULL << (h1 % 64);
  uint64_t w2 = h2 / 64, b2 = 1ULL << (h2 % 64);
  uint64_t w3 = h3 / 64, b3 = 1ULL << (h3 % 64);
  uint64_t p1 = seen[w1]; seen[w1] |= b1;
  uint64_t p2 = seen[w2]; seen[w2] |= b2;
  uint64_t p3 = seen[w3]; seen[w3] |= b3;
  if ((p1 & b1) && (p2 & b2) && (p3 & b3)) {
    solid[w1] |= b1; solid[w2] |= b2; solid[w3] |= b3;
    return true;
  }
  return false;
}

// Twice-tier insert: the same three sequential fetch_or on the seen tier as
// bloom.rs:95-97; every fetch_or that finds its bit already set also sets the
// bit in the twice tier.
bool TwoTierFilter::insert_twice(const Kmer256& km) {
  uint64_t h[3] = {hash_kmer256(km, SEED1) % size_bits, hash_kmer256(km, SEED2) % size_bits,
                   hash_kmer256(km, SEED3) % size_bits};
  bool all = true;
  for (int i = 0; i < 3; i++) {
    uint64_t w = h[i] / 64, b = 1ULL << (h[i] % 64);
    uint64_t p = seen[w];
    seen[w] |= b;
    if (p & b) solid[w] |= b; else all = false;
  }
  return all;
}

// bloom.rs:111-126
bool TwoTierFilter::is_solid_kmer256(const Kmer256& km) const {
  uint64_t h1 = hash_kmer256(km, SEED1) % size_bits;
  uint64_t h2 = hash_kmer256(km, SEED2) % size_bits;
  uint64_t h3 = hash_kmer256(km, SEED3) % size_bits;
  return (solid[h1 / 64] & (1ULL << (h1 % 64))) && (solid[h2 / 64] & (1ULL << (h2 % 64))) &&
         (solid[h3 / 64] & (1ULL << (h3 % 64)));
}

// ---------------------------------------------------------------------------
// src/packed_reads.rs
// ---------------------------------------------------------------------------
// packed_reads.rs:547-578
void PackedReads::pack_clean(const uint8_t* read, size_t len) {
  offsets.push_back(data.size());
  uint32_t clean_len = 0;
  uint8_t byte = 0;
  int shift = 6;
  for (size_t i = 0; i < len; i++) {
    int b2 = base_to_2bit(read[i]);
    if (b2 < 0) continue;  // release-build behaviour: skip non-ACGT
    clean_len++;
    byte |= uint8_t(b2 << shift);
    if (shift == 0) { data.push_back(byte); byte = 0; shift = 6; }
    else shift -= 2;
  }
  if (shift != 6) data.push_back(byte);
  lengths.push_back(clean_len);
}
// packed_reads.rs:592-613
void PackedReads::get_read(size_t idx, std::vector<uint8_t>& buf) const {
  buf.clear();
  size_t len = lengths[idx];
  if (len == 0) return;
  size_t start = offsets[idx], nbytes = (len + 3) / 4, rem = len;
  for (size_t j = 0; j < nbytes; j++) {
    uint8_t byte = data[start + j];
    size_t take = rem < 4 ? rem : 4;
    for (int s = 3; s >= int(4 - take); s--) buf.push_back(bit2_to_base((byte >> (s * 2)) & 3));
    rem -= take;
  }
}
static const size_t MIN_K = 21;  // packed_reads.rs:38
// packed_reads.rs:635-648
static void trim_n_ends(const uint8_t* r, size_t len, size_t* s, size_t* e) {
  size_t a = 0;
  while (a < len && base_to_2bit(r[a]) < 0) a++;
  size_t b = len;
  while (b > 0 && base_to_2bit(r[b - 1]) < 0) b--;
  if (a >= b) { *s = 0; *e = 0; } else { *s = a; *e = b; }
}
// packed_reads.rs:652-654
static bool has_internal_n(const uint8_t* t, size_t len) {
  for (size_t i = 0; i < len; i++) if (base_to_2bit(t[i]) < 0) return true;
  return false;
}
// packed_reads.rs:521-540 (split_on_n packed_reads.rs:659-662)
void PackedReads::ingest_trimmed_unpaired(const uint8_t* t, size_t len) {
  if (len == 0) return;
  bool any = false;
  size_t i = 0;
  while (i < len) {
    while (i < len && base_to_2bit(t[i]) < 0) i++;
    size_t j = i;
    while (j < len && base_to_2bit(t[j]) >= 0) j++;
    if (j > i && j - i >= MIN_K) { pack_clean(t + i, j - i); any = true; }
    i = j;
  }
  if (!any) ambiguous_sidecar.emplace_back((const char*)t, len);
}
// packed_reads.rs:513-517
void PackedReads::ingest_read(const uint8_t* r, size_t len) {
  size_t s, e;
  trim_n_ends(r, len, &s, &e);
  ingest_trimmed_unpaired(r + s, e - s);
}
// packed_reads.rs:291-298
void PackedReads::append_packed(const PackedReads& o) {
  uint64_t base = data.size();
  data.insert(data.end(), o.data.begin(), o.data.end());
  for (uint64_t x : o.offsets) offsets.push_back(x + base);
  lengths.insert(lengths.end(), o.lengths.begin(), o.lengths.end());
  ambiguous_sidecar.insert(ambiguous_sidecar.end(), o.ambiguous_sidecar.begin(),
                           o.ambiguous_sidecar.end());
}
// packed_reads.rs:668-690
static void partition_pair_streaming(const std::string& a, const std::string& b, PackedReads& b1,
                                     PackedReads& b2, PackedReads& b3) {
  const uint8_t* r1 = (const uint8_t*)a.data();
  const uint8_t* r2 = (const uint8_t*)b.data();
  size_t s1, e1, s2, e2;
  trim_n_ends(r1, a.size(), &s1, &e1);
  trim_n_ends(r2, b.size(), &s2, &e2);
  bool n1 = has_internal_n(r1 + s1, e1 - s1), n2 = has_internal_n(r2 + s2, e2 - s2);
  if (!n1 && !n2 && e1 - s1 >= MIN_K && e2 - s2 >= MIN_K) {
    b1.pack_clean(r1 + s1, e1 - s1);
    b2.pack_clean(r2 + s2, e2 - s2);
  } else {
    b3.ingest_trimmed_unpaired(r1 + s1, e1 - s1);
    b3.ingest_trimmed_unpaired(r2 + s2, e2 - s2);
  }
}
// packed_reads.rs:438-461 and finalize_three_blocks packed_reads.rs:481-489
PackedReads from_paired_slices(const std::vector<std::string>& r1,
                               const std::vector<std::string>& r2) {
  PackedReads b1, b2, b3;
  size_t common = std::min(r1.size(), r2.size());
  for (size_t i = 0; i < common; i++) partition_pair_streaming(r1[i], r2[i], b1, b2, b3);
  for (size_t i = common; i < r1.size(); i++) b3.ingest_read((const uint8_t*)r1[i].data(), r1[i].size());
  for (size_t i = common; i < r2.size(); i++) b3.ingest_read((const uint8_t*)r2[i].data(), r2[i].size());
  b1.pe_count = b1.size();
  b1.append_packed(b2);
  b1.append_packed(b3);
  return b1;
}

// packed_reads.rs:69-234 on a memory buffer.  Lines end at '\n' (the last one
// may lack it); next_seq strips every trailing '\n' / '\r' of a line.
bool fastx_records(const uint8_t* text, size_t len, std::vector<std::string>* out, std::string* err) {
  size_t pos = 0;
  // read_until(b'\n'): the next line with its terminator; false at EOF
  auto next_line = [&](size_t* a, size_t* b) {
    if (pos >= len) return false;
    size_t e = pos;
    while (e < len && text[e] != '\n') e++;
    *a = pos;
    *b = e < len ? e + 1 : e;
    pos = *b;
    return true;
  };
  auto strip = [&](size_t a, size_t b) {  // pop trailing \n and \r
    while (b > a && (text[b - 1] == '\n' || text[b - 1] == '\r')) b--;
    return b;
  };
  // open(): skip blank / whitespace-only leading lines (:87-112)
  for (;;) {
    if (pos >= len) return true;  // empty: no records
    const uint8_t c0 = text[pos];
    if (c0 == '\n' || c0 == '\r') {
      size_t a, b;
      next_line(&a, &b);
      continue;
    }
    size_t e = pos;
    while (e < len && text[e] != '\n') e++;
    bool ws = true;
    for (size_t i = pos; i < e; i++) ws &= (text[i] == ' ' || text[i] == '\t' || text[i] == '\r' ||
                                           text[i] == '\x0c');  // u8::is_ascii_whitespace
    if (ws) {
      size_t a, b;
      next_line(&a, &b);
      continue;
    }
    break;
  }
  const bool fastq = text[pos] == '@';
  if (!fastq && text[pos] != '>') {
    *err = "expected '@' or '>' header";
    return false;
  }
  size_t a, b;
  if (!fastq) next_line(&a, &b);  // consume the first '>' header (:118-124)
  for (;;) {
    std::string seq;
    if (fastq) {  // :146-212
      size_t h0, h1;
      for (;;) {
        if (!next_line(&h0, &h1)) return true;
        h1 = strip(h0, h1);
        if (h1 > h0) break;  // blank lines between records are skipped
      }
      if (text[h0] != '@') { *err = "expected '@' header"; return false; }
      size_t s0, s1;
      if (!next_line(&s0, &s1)) { *err = "unexpected EOF waiting for sequence line"; return false; }
      s1 = strip(s0, s1);
      seq.assign((const char*)text + s0, s1 - s0);
      size_t p0, p1;
      if (!next_line(&p0, &p1)) { *err = "unexpected EOF waiting for '+' separator"; return false; }
      if (p1 == p0 || text[p0] != '+') { *err = "expected '+' separator line"; return false; }
      size_t q0, q1;
      if (!next_line(&q0, &q1)) { *err = "unexpected EOF waiting for quality scores"; return false; }
      q1 = strip(q0, q1);
      if (q1 - q0 != seq.size()) { *err = "sequence length != quality length"; return false; }
      out->push_back(std::move(seq));
    } else {  // :214-231
      for (;;) {
        size_t l0, l1;
        if (!next_line(&l0, &l1)) {
          if (!seq.empty()) out->push_back(std::move(seq));
          return true;
        }
        l1 = strip(l0, l1);
        if (l1 > l0 && text[l0] == '>') break;
        seq.append((const char*)text + l0, l1 - l0);
      }
      out->push_back(std::move(seq));
    }
  }
}

bool from_paired_texts(const uint8_t* t1, size_t l1, const uint8_t* t2, size_t l2, PackedReads* out,
                       std::string* err) {
  std::vector<std::string> a, b;
  if (!fastx_records(t1, l1, &a, err) || !fastx_records(t2, l2, &b, err)) return false;
  *out = from_paired_slices(a, b);  // pairs, then the longer file's tail into Block 3
  return true;
}

bool from_single_text(const uint8_t* t, size_t l, PackedReads* out, std::string* err) {
  std::vector<std::string> a;
  if (!fastx_records(t, l, &a, err)) return false;
  *out = PackedReads();
  for (auto& r : a) out->ingest_read((const uint8_t*)r.data(), r.size());
  return true;
}

// ---------------------------------------------------------------------------
// Count map: open addressing with linear probing, grown at 7/8 load like
// hashbrown's maximum load factor.  Storage only: its hash never reaches any
// output because every output is sorted by key.
// ---------------------------------------------------------------------------
struct KmerMap {
  std::vector<Kmer256> keys;
  std::vector<uint32_t> vals;
  std::vector<uint8_t> used;
  size_t mask = 0, n = 0;
  explicit KmerMap(size_t cap = 16) { reset(cap); }
  void reset(size_t cap) {
    size_t c = 16;
    while (c * 7 / 8 < cap) c <<= 1;
    keys.assign(c, Kmer256());
    vals.assign(c, 0);
    used.assign(c, 0);
    mask = c - 1;
    n = 0;
  }
  static inline uint64_t mix(const Kmer256& k) {
    uint64_t a = (uint64_t)k.lo ^ ((uint64_t)(k.lo >> 64) * 0x9e3779b97f4a7c15ULL) ^
                 ((uint64_t)k.hi * 0xc2b2ae3d27d4eb4fULL) ^ ((uint64_t)(k.hi >> 64) * 0x165667b19e3779f9ULL);
    a ^= a >> 31; a *= 0xbf58476d1ce4e5b9ULL; a ^= a >> 29;
    return a;
  }
  void grow() {
    std::vector<Kmer256> ok; std::vector<uint32_t> ov; std::vector<uint8_t> ou;
    ok.swap(keys); ov.swap(vals); ou.swap(used);
    size_t c = (mask + 1) * 2;
    keys.assign(c, Kmer256()); vals.assign(c, 0); used.assign(c, 0);
    mask = c - 1; n = 0;
    for (size_t i = 0; i < ok.size(); i++) if (ou[i]) add(ok[i], ov[i]);
  }
  inline void add(const Kmer256& k, uint32_t v) {
    if ((n + 1) * 8 > (mask + 1) * 7) grow();
    size_t i = mix(k) & mask;
    while (used[i]) {
      if (keys[i] == k) { vals[i] += v; return; }
      i = (i + 1) & mask;
    }
    used[i] = 1; keys[i] = k; vals[i] = v; n++;
  }
  void drain_into(std::vector<CountEntry>& out) const {
    for (size_t i = 0; i <= mask; i++) if (used[i]) out.push_back(CountEntry{keys[i], vals[i]});
  }
};

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static void sort_entries(std::vector<CountEntry>& v) {
  std::sort(v.begin(), v.end(), [](const CountEntry& a, const CountEntry& b) { return a.key < b.key; });
}

// assemble.rs:129-161 (Stage 2) and 166-242 (Stage 3), serial order.
void count_serial(const PackedReads& pr, unsigned k, uint64_t bloom_bits, Mode mode,
                  CountResult* out, bool correct) {
  double t0 = now_s();
  TwoTierFilter f(bloom_bits);
  std::vector<uint8_t> buf;
  uint64_t occ = 0;
  for (size_t idx = 0; idx < pr.size(); idx++) {
    pr.get_read(idx, buf);
    if (buf.size() < k) continue;
    for (size_t i = 0; i + k <= buf.size(); i++) {
      Kmer256 km;
      if (k256_from_bytes(buf.data() + i, k, k, &km)) {
        Kmer256 can = k256_canonical(km, k, nullptr);
        if (mode == MODE_REF) f.insert_kmer256(can); else f.insert_twice(can);
        occ++;
      }
    }
  }
  double t1 = now_s();
  KmerMap map(1024);
  uint64_t adm = 0, ncorr = 0;
  for (size_t idx = 0; idx < pr.size(); idx++) {
    pr.get_read(idx, buf);
    if (buf.size() < k) continue;
    if (correct && correct_read_in_place(k, buf, f)) ncorr++;  // assemble.rs:188-191
    for (size_t i = 0; i + k <= buf.size(); i++) {
      Kmer256 km;
      if (k256_from_bytes(buf.data() + i, k, k, &km)) {
        Kmer256 can = k256_canonical(km, k, nullptr);
        if (f.is_solid_kmer256(can)) { map.add(can, 1); adm++; }
      }
    }
  }
  double t2 = now_s();
  out->table.clear();
  map.drain_into(out->table);
  sort_entries(out->table);
  out->seen = f.seen;
  out->solid = f.solid;
  out->occurrences = occ;
  out->admitted_occurrences = adm;
  out->corrected_reads = ncorr;
  out->seconds_stage2 = t1 - t0;
  out->seconds_stage3 = t2 - t1;
  out->seconds_total = now_s() - t0;
}

// Threaded restatement (CPU baseline).  Chunking assemble.rs:137-139; rayon's
// dynamic chunk scheduling is modelled by an atomic chunk cursor.
void count_threaded(const PackedReads& pr, unsigned k, uint64_t bloom_bits, int threads,
                    Mode mode, bool keep_bloom, CountResult* out, bool correct, size_t stage3_reads) {
  double t0 = now_s();
  if (threads < 1) threads = 1;
  uint64_t num_words = (bloom_bits + 63) / 64;
  if (num_words < 1) num_words = 1;
  uint64_t size_bits = num_words * 64;
  std::vector<std::atomic<uint64_t>> seen(num_words), solid(num_words);
  for (uint64_t i = 0; i < num_words; i++) { seen[i].store(0, std::memory_order_relaxed); solid[i].store(0, std::memory_order_relaxed); }

  size_t n = pr.size();
  size_t chunk = std::max<size_t>(n / size_t(threads), 1000);  // assemble.rs:138
  size_t num_chunks = (n + chunk - 1) / chunk;                  // assemble.rs:139
  std::atomic<size_t> cursor{0};
  std::atomic<uint64_t> occ_total{0};

  auto hash3 = [&](const Kmer256& c, uint64_t* w, uint64_t* b) {
    uint64_t h1 = hash_kmer256(c, SEED1) % size_bits;
    uint64_t h2 = hash_kmer256(c, SEED2) % size_bits;
    uint64_t h3 = hash_kmer256(c, SEED3) % size_bits;
    w[0] = h1 / 64; b[0] = 1ULL << (h1 % 64);
    w[1] = h2 / 64; b[1] = 1ULL << (h2 % 64);
    w[2] = h3 / 64; b[2] = 1ULL << (h3 % 64);
  };

  // Stage 2 (assemble.rs:141-157)
  auto stage2 = [&]() {
    std::vector<uint8_t> buf;
    buf.reserve(512);
    uint64_t occ = 0;
    for (;;) {
      size_t c = cursor.fetch_add(1);
      if (c >= num_chunks) break;
      size_t start = c * chunk, end = std::min(start + chunk, n);
      for (size_t idx = start; idx < end; idx++) {
        pr.get_read(idx, buf);
        if (buf.size() < k) continue;
        for (size_t i = 0; i + k <= buf.size(); i++) {
          Kmer256 km;
          if (!k256_from_bytes(buf.data() + i, k, k, &km)) continue;
          Kmer256 can = k256_canonical(km, k, nullptr);
          uint64_t w[3], b[3];
          hash3(can, w, b);
          occ++;
          if (mode == MODE_REF) {  // bloom.rs:95-106
            uint64_t p1 = seen[w[0]].fetch_or(b[0], std::memory_order_relaxed);
            uint64_t p2 = seen[w[1]].fetch_or(b[1], std::memory_order_relaxed);
            uint64_t p3 = seen[w[2]].fetch_or(b[2], std::memory_order_relaxed);
            if ((p1 & b[0]) && (p2 & b[1]) && (p3 & b[2])) {
              solid[w[0]].fetch_or(b[0], std::memory_order_relaxed);
              solid[w[1]].fetch_or(b[1], std::memory_order_relaxed);
              solid[w[2]].fetch_or(b[2], std::memory_order_relaxed);
            }
          } else {
            for (int j = 0; j < 3; j++) {
              uint64_t p = seen[w[j]].fetch_or(b[j], std::memory_order_relaxed);
              if (p & b[j]) solid[w[j]].fetch_or(b[j], std::memory_order_relaxed);
            }
          }
        }
      }
    }
    occ_total.fetch_add(occ);
  };
  {
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++) ts.emplace_back(stage2);
    for (auto& t : ts) t.join();
  }
  double t1 = now_s();

  // Stage 3 (assemble.rs:166-219)
  size_t num_shards = 1;
  while (num_shards < size_t(threads) * 4) num_shards <<= 1;
  num_shards = std::min<size_t>(std::max<size_t>(num_shards, 8), 64);  // assemble.rs:167
  size_t shard_mask = num_shards - 1;
  // config.error_correct (assemble.rs:183-191): the corrector reads the
  // filter through a plain snapshot of the finished tiers.
  TwoTierFilter snap(correct ? size_bits : 64);
  if (correct)
    for (uint64_t i = 0; i < num_words; i++) snap.solid[i] = solid[i].load(std::memory_order_relaxed);
  std::atomic<uint64_t> corr_total{0};
  std::vector<std::mutex> locks(num_shards);
  std::vector<KmerMap> shards;
  for (size_t s = 0; s < num_shards; s++) shards.emplace_back(75000);  // assemble.rs:170
  std::atomic<uint64_t> adm_total{0};
  cursor.store(0);
  // stage3_reads < n: Stage 3 over the first stage3_reads reads only (a timed
  // sample of the full Stage 3 against the full filter)
  const size_t n3 = std::min(n, stage3_reads);
  const size_t chunk3 = std::min(chunk, std::max<size_t>(n3 / size_t(threads), 1));
  const size_t num_chunks3 = n3 ? (n3 + chunk3 - 1) / chunk3 : 0;
  auto stage3 = [&]() {
    std::vector<uint8_t> buf;
    buf.reserve(512);
    uint64_t adm = 0;
    for (;;) {
      size_t c = cursor.fetch_add(1);
      if (c >= num_chunks3) break;
      size_t start = c * chunk3, end = std::min(start + chunk3, n3);
      std::vector<std::vector<Kmer256>> tb(num_shards);
      for (auto& v : tb) v.reserve(256);
      for (size_t idx = start; idx < end; idx++) {
        pr.get_read(idx, buf);
        if (buf.size() < k) continue;
        if (correct && correct_read_in_place(k, buf, snap)) corr_total.fetch_add(1);
        for (size_t i = 0; i + k <= buf.size(); i++) {
          Kmer256 km;
          if (!k256_from_bytes(buf.data() + i, k, k, &km)) continue;
          Kmer256 can = k256_canonical(km, k, nullptr);
          uint64_t w[3], b[3];
          hash3(can, w, b);
          bool ok = (solid[w[0]].load(std::memory_order_relaxed) & b[0]) &&
                    (solid[w[1]].load(std::memory_order_relaxed) & b[1]) &&
                    (solid[w[2]].load(std::memory_order_relaxed) & b[2]);
          if (!ok) continue;
          adm++;
          size_t si = size_t((uint64_t)can.lo) & shard_mask;  // assemble.rs:197
          tb[si].push_back(can);
          if (tb[si].size() >= 256) {                          // assemble.rs:199-204
            std::lock_guard<std::mutex> g(locks[si]);
            for (auto& x : tb[si]) shards[si].add(x, 1);
            tb[si].clear();
          }
        }
      }
      for (size_t si = 0; si < num_shards; si++) {             // assemble.rs:211-218
        if (tb[si].empty()) continue;
        std::lock_guard<std::mutex> g(locks[si]);
        for (auto& x : tb[si]) shards[si].add(x, 1);
        tb[si].clear();
      }
    }
    adm_total.fetch_add(adm);
  };
  {
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++) ts.emplace_back(stage3);
    for (auto& t : ts) t.join();
  }
  double t2 = now_s();
  // Merge (assemble.rs:238-242); shards hold disjoint keys.
  out->table.clear();
  out->table.reserve(5000000);
  for (auto& s : shards) s.drain_into(out->table);
  sort_entries(out->table);
  if (keep_bloom) {
    out->seen.resize(num_words);
    out->solid.resize(num_words);
    for (uint64_t i = 0; i < num_words; i++) {
      out->seen[i] = seen[i].load();
      out->solid[i] = solid[i].load();
    }
  } else {
    out->seen.clear();
    out->solid.clear();
  }
  out->occurrences = occ_total.load();
  out->admitted_occurrences = adm_total.load();
  out->corrected_reads = corr_total.load();
  out->seconds_stage2 = t1 - t0;
  out->seconds_stage3 = t2 - t1;
  out->seconds_total = now_s() - t0;
}

// assemble.rs:692-735
uint32_t determine_solid_kmer_cutoff(const std::vector<uint32_t>& counts, double min_coverage) {
  if (min_coverage > 5.0) {
    double v = std::max(min_coverage * 0.35, 2.0);
    if (!(v >= 0)) return 0;
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return uint32_t(v);
  }
  if (counts.size() <= 100) return 2;
  std::vector<uint32_t> s(counts);
  std::sort(s.begin(), s.end());
  uint32_t top_cov = s[s.size() * 95 / 100];
  if (top_cov < 30) return 2;
  uint32_t mvs = std::min<uint32_t>(std::max<uint32_t>(top_cov / 4, 10), 35);
  std::vector<size_t> hist(mvs + 1, 0);
  for (uint32_t c : s) if (c <= mvs) hist[c]++;
  uint32_t valley = 2;
  size_t min_val = SIZE_MAX;
  bool found = false;
  for (uint32_t c = 2; c <= mvs; c++) {
    size_t h = hist[c];
    if (h <= min_val) { min_val = h; valley = c; }
    else if (h > min_val * 2 && c > valley + 2) { found = true; break; }
  }
  return found ? valley : 2;
}

// (k+1)-mer produced by appending base b to the k-mer x (both Kmer256 layout).
static Kmer256 append_base(const Kmer256& x, uint8_t b, unsigned k) {
  Kmer256 r;
  if (k + 1 <= 64) { r.lo = (x.lo << 2) | (u128)(b & 3); return r; }
  if (k == 64) { r.lo = x.lo; r.hi = (u128)(b & 3); return r; }
  r.lo = x.lo;
  r.hi = (x.hi << 2) | (u128)(b & 3);
  return r;
}

// graph.rs:78-89 get_successors with OrientedKmer::explicit_seq graph.rs:24-30,
// enumerated over both orientations of every solid k-mer.  Each successor
// relation s -> t is the (k+1)-mer explicit(s)+b; the set of their canonical
// forms is the edge list.
std::vector<Kmer256> edges(const std::vector<Kmer256>& solid_sorted, unsigned k) {
  std::vector<Kmer256> out;
  auto is_solid = [&](const Kmer256& x) {
    return std::binary_search(solid_sorted.begin(), solid_sorted.end(), x);
  };
  for (const Kmer256& s : solid_sorted) {
    for (int o = 0; o < 2; o++) {
      Kmer256 ex = o ? k256_revcomp(s, k) : s;
      for (uint8_t b = 0; b < 4; b++) {
        Kmer256 nx = k256_extend_right(ex, b, k);
        Kmer256 can = k256_canonical(nx, k, nullptr);
        if (!is_solid(can)) continue;
        Kmer256 e = append_base(ex, b, k);
        out.push_back(k256_canonical(e, k + 1, nullptr));
      }
    }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

// src/assemble.rs:267-283
void inject_priors(CountResult* r, const std::vector<std::vector<uint8_t>>& priors, unsigned k,
                   uint32_t boost) {
  std::map<Kmer256, uint32_t> m;  // ordered by Kmer256 (lexicographic on (lo, hi))
  for (const auto& e : r->table) m[e.key] = e.count;
  for (const auto& seq : priors) {
    if (seq.size() < k) continue;                      // :273-275
    for (size_t i = 0; i + k <= seq.size(); i++) {     // :276
      Kmer256 x;
      if (!k256_from_bytes(seq.data() + i, k, k, &x)) continue;  // :277
      bool rc;
      m[k256_canonical(x, k, &rc)] += boost;           // :278-279
    }
  }
  r->table.clear();
  for (const auto& kv : m) r->table.push_back(CountEntry{kv.first, kv.second});
}

// src/graph.rs:14-40, 65-235
namespace {
struct OK {
  Kmer256 kmer;
  bool is_rc;
};
}  // namespace

std::vector<Unitig> unitigs(const std::vector<Kmer256>& solid, const std::vector<uint32_t>& counts,
                            unsigned k) {
  std::vector<Unitig> out;
  if (k == 0 || solid.empty()) return out;  // :70-75
  auto index_of = [&](const Kmer256& x) -> long {
    auto it = std::lower_bound(solid.begin(), solid.end(), x);
    return (it != solid.end() && *it == x) ? (long)(it - solid.begin()) : -1;
  };
  auto explicit_seq = [&](const OK& o) { return o.is_rc ? k256_revcomp(o.kmer, k) : o.kmer; };  // :24-30
  auto succs = [&](const OK& o) {  // :78-90
    std::vector<OK> v;
    const Kmer256 s = explicit_seq(o);
    for (uint8_t b = 0; b < 4; b++) {
      bool rc;
      const Kmer256 can = k256_canonical(k256_extend_right(s, b, k), k, &rc);
      if (index_of(can) >= 0) v.push_back(OK{can, rc});
    }
    return v;
  };
  auto preds = [&](const OK& o) {  // :91-102
    std::vector<OK> v;
    const Kmer256 s = explicit_seq(o);
    for (uint8_t a = 0; a < 4; a++) {
      bool rc;
      const Kmer256 can = k256_canonical(k256_prepend_left(s, a, k), k, &rc);
      if (index_of(can) >= 0) v.push_back(OK{can, rc});
    }
    return v;
  };
  std::vector<char> visited(solid.size(), 0);
  auto vis = [&](const Kmer256& x) { return visited[index_of(x)] != 0; };
  auto mark = [&](const Kmer256& x) { visited[index_of(x)] = 1; };
  auto extract = [&](OK start) {  // :104-157
    std::vector<OK> path;
    OK curr = start;
    while (!vis(curr.kmer)) {
      mark(curr.kmer);
      path.push_back(curr);
      const auto sc = succs(curr);
      if (sc.size() != 1) break;
      const OK nx = sc[0];
      if (vis(nx.kmer)) break;
      if (preds(nx).size() != 1) break;
      curr = nx;
    }
    if (path.empty()) return path;
    std::vector<OK> back;
    OK bc = path[0];
    for (;;) {
      const auto pr = preds(bc);
      if (pr.size() != 1) break;
      const OK pv = pr[0];
      if (vis(pv.kmer)) break;
      if (succs(pv).size() != 1) break;
      mark(pv.kmer);
      back.push_back(pv);
      bc = pv;
    }
    std::reverse(back.begin(), back.end());
    back.insert(back.end(), path.begin(), path.end());
    return back;
  };
  auto build = [&](const std::vector<OK>& path) {  // :159-177
    std::string seq = k256_to_string(explicit_seq(path[0]), k);
    double cov = (double)counts[index_of(path[0].kmer)];
    for (size_t i = 1; i < path.size(); i++) {
      const Kmer256 e = explicit_seq(path[i]);
      seq.push_back("ACGT"[k256_last_base(e, k)]);
      cov += (double)counts[index_of(path[i].kmer)];
    }
    return Unitig{seq, cov / (double)path.size(), path.size()};
  };
  for (const Kmer256& km : solid) {  // pass 1, :183-216
    if (vis(km)) continue;
    OK start{km, false};
    const auto pf = preds(start);
    const auto pr = preds(OK{km, true});
    if (pf.size() == 1) {
      const OK pn = pf[0];
      if (succs(pn).size() == 1 && !vis(pn.kmer)) {
        if (pr.size() == 1) {
          const OK prn = pr[0];
          if (succs(prn).size() == 1 && !vis(prn.kmer)) continue;  // interior: deferred
          start = OK{km, true};
        } else {
          start = OK{km, true};
        }
      }
    }
    const auto p = extract(start);
    if (!p.empty()) out.push_back(build(p));
  }
  for (const Kmer256& km : solid) {  // pass 2, :219-231
    if (vis(km)) continue;
    const auto p = extract(OK{km, false});
    if (!p.empty()) out.push_back(build(p));
  }
  // orientation not greater than the reverse complement; sorted by sequence
  for (Unitig& u : out) {
    std::string rc(u.sequence.rbegin(), u.sequence.rend());
    for (char& c : rc) c = c == 'A' ? 'T' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'A';
    if (rc < u.sequence) u.sequence = rc;
  }
  std::sort(out.begin(), out.end(), [](const Unitig& a, const Unitig& b) { return a.sequence < b.sequence; });
  return out;
}

// ---------------------------------------------------------------------------
// src/hammer.rs
// ---------------------------------------------------------------------------
bool correct_read_in_place(unsigned k, std::vector<uint8_t>& seq, const TwoTierFilter& filter) {
  if (k == 0 || k > 128 || seq.size() < k) return false;  // :41-43
  std::vector<uint8_t> scratch(seq);                      // :45-46
  bool modified = false;
  const size_t n = scratch.size();
  // from_bytes + canonical + is_solid_kmer256 of the window at s; None is not solid
  auto solid_at = [&](size_t s) {
    Kmer256 km;
    if (!k256_from_bytes(scratch.data() + s, k, k, &km)) return false;
    return filter.is_solid_kmer256(k256_canonical(km, k, nullptr));
  };
  for (size_t i = 0; i + k <= n; i++) {  // :49
    Kmer256 km;
    if (!k256_from_bytes(scratch.data() + i, k, k, &km)) continue;  // :50
    if (filter.is_solid_kmer256(k256_canonical(km, k, nullptr))) continue;  // :51-52
    bool have = false;
    size_t best_off = 0;
    uint8_t best_base = 0;
    size_t max_gain = 0;
    for (size_t offset = 0; offset < k; offset++) {  // :56
      const size_t pos = i + offset;
      const uint8_t orig = scratch[pos];
      const uint8_t orig_upper = (orig >= 'a' && orig <= 'z') ? (uint8_t)(orig - 32) : orig;
      const size_t start_scan = pos >= k - 1 ? pos - (k - 1) : 0;  // :60
      const size_t end_scan = std::min(pos, n - k);                 // :61
      size_t base_solid = 0;  // :63-74
      for (size_t s = start_scan; s <= end_scan; s++)
        if (s != i && solid_at(s)) base_solid++;
      for (uint8_t cand : {(uint8_t)'A', (uint8_t)'C', (uint8_t)'G', (uint8_t)'T'}) {  // :76
        if (cand == orig_upper) continue;
        scratch[pos] = cand;
        if (solid_at(i)) {  // :81-84
          size_t solid_count = 1;
          for (size_t s = start_scan; s <= end_scan; s++)
            if (s != i && solid_at(s)) solid_count++;
          const size_t gain = solid_count > base_solid ? solid_count - base_solid : 0;  // :99
          if (gain > max_gain) {  // :100-103
            max_gain = gain;
            have = true;
            best_off = offset;
            best_base = cand;
          }
        }
        scratch[pos] = orig;  // :106
      }
    }
    if (have) {  // :111-115
      seq[i + best_off] = best_base;
      scratch[i + best_off] = best_base;
      modified = true;
    }
  }
  return modified;
}

}  // namespace ora
