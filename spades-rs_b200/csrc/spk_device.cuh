// spk_device.cuh -- device primitives for canonical k-mers on packed reads.
//
// A k-mer is held as its 2k-bit "sequence value" V: base 0 in the two most
// significant bits of the 2k-bit number, little-endian 64-bit limbs, NL =
// ceil(k/32) limbs.  For k <= 64 V is exactly the reference Kmer256.lo
// (src/dna.rs:299-321); for k > 64 Kmer256 = (V >> 2(k-64), V & mask) and the
// lexicographic Kmer256 order (src/dna.rs:137) equals the numeric order of V,
// so canonical selection, table keys and sorting all work on V.
#pragma once
#include <cstdint>

namespace spk {

constexpr uint64_t kSeed1 = 0x517cc1b727220a95ULL;  // src/bloom.rs:84
constexpr uint64_t kSeed2 = 0x9e3779b97f4a7c15ULL;  // src/bloom.rs:85
constexpr uint64_t kSeed3 = 0x6c62272e07bb0142ULL;  // src/bloom.rs:86
constexpr uint64_t kM55 = 0x5555555555555555ULL;

template <int NL>
struct Seq {
  uint64_t v[NL];
};

__device__ __forceinline__ uint64_t bswap64(uint64_t x) {
  uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
  uint32_t a = __byte_perm(lo, 0, 0x0123), b = __byte_perm(hi, 0, 0x0123);
  return ((uint64_t)a << 32) | b;
}
// (hi:lo) << s, top 64 bits, for 0 <= s <= 63.
__device__ __forceinline__ uint64_t shl2(uint64_t hi, uint64_t lo, unsigned s) {
  return (hi << s) | ((lo >> 1) >> (63 - s));
}
// (hi:lo) >> s, low 64 bits, for 0 <= s <= 63.
__device__ __forceinline__ uint64_t shr2(uint64_t hi, uint64_t lo, unsigned s) {
  return (lo >> s) | ((hi << 1) << (63 - s));
}
__device__ __forceinline__ uint64_t rotl64(uint64_t x, unsigned r) {
  return (x << r) | (x >> (64 - r));
}

// Window of 2k bits starting at big-endian bit offset `bitpos` of the packed
// byte stream (base i of a read at byte offset o is at bit 8*o + 2*i).  The
// buffer must be readable for 8*(NL+1) bytes past the word holding bitpos.
template <int NL>
__device__ __forceinline__ Seq<NL> extract(const uint64_t* __restrict__ words, uint64_t bitpos,
                                           unsigned k) {
  const uint64_t* p = words + (bitpos >> 6);
  const unsigned s = (unsigned)(bitpos & 63);
  uint64_t U[NL + 1];
#pragma unroll
  for (int j = 0; j <= NL; j++) U[j] = bswap64(__ldg(p + j));
  uint64_t X[NL];  // X[NL-1] most significant
#pragma unroll
  for (int j = 0; j < NL; j++) X[NL - 1 - j] = shl2(U[j], U[j + 1], s);
  const unsigned r = 64u * NL - 2u * k;  // 0 <= r < 64
  Seq<NL> V;
#pragma unroll
  for (int i = 0; i < NL; i++) V.v[i] = (i + 1 < NL) ? shr2(X[i + 1], X[i], r) : (X[i] >> r);
  return V;
}

// Reverse complement of a 2k-bit sequence value (src/dna.rs:65-78, 118-132,
// 152-180): complement every base and reverse the base order.
template <int NL>
__device__ __forceinline__ Seq<NL> revcomp(const Seq<NL>& V, unsigned k) {
  uint64_t B[NL];
#pragma unroll
  for (int i = 0; i < NL; i++) {
    uint64_t x = __brevll(~V.v[NL - 1 - i]);
    B[i] = ((x >> 1) & kM55) | ((x & kM55) << 1);
  }
  const unsigned r = 64u * NL - 2u * k;
  Seq<NL> R;
#pragma unroll
  for (int i = 0; i < NL; i++) R.v[i] = (i + 1 < NL) ? shr2(B[i + 1], B[i], r) : (B[i] >> r);
  return R;
}

template <int NL>
__device__ __forceinline__ bool seq_le(const Seq<NL>& a, const Seq<NL>& b) {
#pragma unroll
  for (int i = NL - 1; i >= 0; i--) {
    if (a.v[i] != b.v[i]) return a.v[i] < b.v[i];
  }
  return true;
}
template <int NL>
__device__ __forceinline__ bool seq_eq(const Seq<NL>& a, const Seq<NL>& b) {
  bool e = true;
#pragma unroll
  for (int i = 0; i < NL; i++) e &= a.v[i] == b.v[i];
  return e;
}

// Canonical k-mer (src/dna.rs:185-192): min(fwd, rc), ties keep fwd.
template <int NL>
__device__ __forceinline__ Seq<NL> canonical(const Seq<NL>& V, unsigned k, bool* is_rc = nullptr) {
  Seq<NL> R = revcomp<NL>(V, k);
  bool f = seq_le<NL>(V, R);
  if (is_rc) *is_rc = !f;
  return f ? V : R;
}

// X.extend_right(b) (src/dna.rs:196-221): drop the first base, append b.
template <int NL>
__device__ __forceinline__ Seq<NL> shl_append(const Seq<NL>& X, unsigned b, unsigned k) {
  Seq<NL> R;
#pragma unroll
  for (int i = NL - 1; i >= 1; i--) R.v[i] = shl2(X.v[i], X.v[i - 1], 2);
  R.v[0] = (X.v[0] << 2) | b;
  const unsigned topbits = 2u * k - 64u * (NL - 1);  // bits used in the top limb (1..64)
  if (topbits < 64) R.v[NL - 1] &= (1ULL << topbits) - 1;
  return R;
}
// The reverse complement of X.extend_right(b), from RC = revcomp(X): the
// complement of b enters at the front (the top two of the 2k bits) and the
// last base of RC drops out.
template <int NL>
__device__ __forceinline__ Seq<NL> shr_prepend(const Seq<NL>& RC, unsigned c, unsigned k) {
  Seq<NL> R;
#pragma unroll
  for (int i = 0; i < NL; i++) R.v[i] = (i + 1 < NL) ? shr2(RC.v[i + 1], RC.v[i], 2) : (RC.v[i] >> 2);
  const unsigned top = 2u * k - 2u;  // bit of the first base
#pragma unroll
  for (int i = 0; i < NL; i++)
    if ((unsigned)i == (top >> 6)) R.v[i] |= (uint64_t)c << (top & 63);
  return R;
}

// 64 bits of V starting at bit b (bits above the value read as zero).
template <int NL>
__device__ __forceinline__ uint64_t bits64(const Seq<NL>& V, unsigned b) {
  const unsigned i = b >> 6, s = b & 63;
  uint64_t lo = 0, hi = 0;
#pragma unroll
  for (int j = 0; j < NL; j++) {
    if ((unsigned)j == i) lo = V.v[j];
    if ((unsigned)j == i + 1) hi = V.v[j];
  }
  return shr2(hi, lo, s);
}

// The four u64 limbs of the reference Kmer256 (src/bloom.rs:62-65).
template <int NL>
__device__ __forceinline__ void kmer256_limbs(const Seq<NL>& V, unsigned k, uint64_t w[4]) {
  if (NL <= 2) {
    w[0] = V.v[0];
    w[1] = NL == 2 ? V.v[NL - 1] : 0;
    w[2] = 0;
    w[3] = 0;
  } else {
    const unsigned t = 2u * (k - 64);  // bits held in Kmer256.hi
    w[0] = bits64<NL>(V, t);
    w[1] = bits64<NL>(V, t + 64);
    const uint64_t v0 = V.v[0], v1 = V.v[1];
    w[2] = t >= 64 ? v0 : (v0 & ((1ULL << t) - 1));
    w[3] = t > 64 ? (v1 & ((1ULL << (t - 64)) - 1)) : 0;
  }
}

// hash_kmer256 (src/bloom.rs:61-78) split into the seed-independent limb
// products and the per-seed mixing chain.
struct HashPre {
  uint64_t w0, p1, p2, p3;
};
__device__ __forceinline__ HashPre hash_pre(const uint64_t w[4]) {
  HashPre h;
  h.w0 = w[0];
  h.p1 = rotl64(w[1], 21) * 0x9e3779b97f4a7c15ULL;
  h.p2 = rotl64(w[2], 43) * 0xbf58476d1ce4e5b9ULL;
  h.p3 = rotl64(w[3], 11) * 0x94d049bb133111ebULL;
  return h;
}
__device__ __forceinline__ uint64_t hash_seed(const HashPre& h, uint64_t seed) {
  uint64_t x = h.w0 ^ seed;
  x = (x ^ h.p1) * 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x = (x ^ h.p2) * 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  x = (x ^ h.p3) * 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  return x;
}

// `h % d` for a divisor fixed per filter (src/bloom.rs:84-86 take
// hash % size_bits).  Powers of two use a mask; other divisors use the
// unsigned division by an invariant integer of Granlund & Montgomery,
// "Division by Invariant Integers using Multiplication" (PLDI 1994), Fig. 4.1
// with N = 64.  The host computes the constants (FastMod::make).
struct FastMod {
  uint64_t d, mask, mprime;
  uint32_t sh1, sh2, pow2, pad;
};
__device__ __forceinline__ uint64_t fastmod(const FastMod& f, uint64_t n) {
  if (f.pow2) return n & f.mask;
  uint64_t t1 = __umul64hi(f.mprime, n);
  uint64_t q = (t1 + ((n - t1) >> f.sh1)) >> f.sh2;
  return n - q * f.d;
}

// Exclusive lane mask below the calling lane.
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

}  // namespace spk
