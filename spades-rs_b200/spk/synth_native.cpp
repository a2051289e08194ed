// synth_native.cpp -- seeded synthetic read sets for the batched and serving
// workloads, written straight into the PackedReads layout
// (src/packed_reads.rs:42-59, 547-578).  Host C++ (no CUDA): the Python
// generator in synth.py takes minutes for the tens of Gbp those workloads
// name, this one seconds.
//
// Every random draw is a pure function of (seed, stream, counter) through
// splitmix64 (Steele, Lea & Flood 2014), so the output does not depend on
// the thread count.  A genome base is drawn from its position; a read pair
// from its index: fragment length ~ N(mean, sd) by Box-Muller, a uniform
// start, a uniform strand, and per-base substitutions to a uniform other base.
// Reads are N-free and of one length, so every pair is clean: block 1 holds
// the mates 1 in pair order and block 2 the mates 2 in the same order, each
// read starting on a byte boundary with its first base in the top bits of
// its first byte.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

// A counter-based stream: draw j of stream (seed, stream, item).
struct Rng {
  uint64_t key;
  uint64_t ctr = 0;
  Rng(uint64_t seed, uint64_t stream, uint64_t item)
      : key(splitmix64(splitmix64(seed * 0x100000001b3ULL ^ stream) ^ item * 0xd6e8feb86659fd93ULL)) {}
  uint64_t next() { return splitmix64(key + 0x632be59bd9b4e019ULL * ++ctr); }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)
  double normal() {
    const double u1 = 1.0 - uniform(), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

template <class F>
void parallel_for(uint64_t n, int threads, F f) {
  if (threads < 1) threads = 1;
  const uint64_t per = (n + threads - 1) / threads;
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; t++) {
    const uint64_t a = t * per, b = std::min<uint64_t>(n, a + per);
    if (a >= b) break;
    ts.emplace_back([=] { f(a, b); });
  }
  for (auto& t : ts) t.join();
}

}  // namespace

extern "C" {

// A genome of `len` bases, codes 0..3 (A C G T), P(C) = P(G) = gc / 2.
void spk_synth_genome(uint8_t* out, uint64_t len, double gc, uint64_t seed, uint64_t stream, int threads) {
  const double pa = (1.0 - gc) / 2, pc = pa + gc / 2, pg = pc + gc / 2;
  parallel_for((len + 4095) / 4096, threads, [&](uint64_t a, uint64_t b) {
    for (uint64_t blk = a; blk < b; blk++) {
      Rng r(seed, stream, blk);
      const uint64_t e = std::min<uint64_t>(len, (blk + 1) * 4096);
      for (uint64_t i = blk * 4096; i < e; i++) {
        const double u = r.uniform();
        out[i] = u < pa ? 0 : u < pc ? 1 : u < pg ? 2 : 3;
      }
    }
  });
}

// n_pairs clean 2 x read_len pairs from `genome` (codes), written as packed
// reads of ceil(read_len / 4) bytes each: mate 1 of pair i is read first1 +
// i, mate 2 is read first2 + i, and read j starts at byte j * that size (the
// store of a read set whose reads all have this length).  Pair i draws from
// stream (seed, stream, i).  err: substitution probability per base.
void spk_synth_pairs(const uint8_t* genome, uint64_t glen, uint64_t n_pairs, uint32_t read_len,
                     double frag_mean, double frag_sd, double err, uint64_t seed, uint64_t stream,
                     uint64_t first1, uint64_t first2, uint8_t* data, uint64_t* offsets, uint32_t* lengths,
                     int threads) {
  const uint64_t nb = (read_len + 3) / 4;
  parallel_for(n_pairs, threads, [&](uint64_t a, uint64_t b) {
    std::vector<uint8_t> r1(read_len), r2(read_len);
    for (uint64_t i = a; i < b; i++) {
      Rng r(seed, stream, i);
      double f = std::nearbyint(frag_mean + frag_sd * r.normal());
      uint64_t frag = f < read_len ? read_len : (uint64_t)f;
      if (frag > glen) frag = glen;
      const uint64_t start = (uint64_t)(r.uniform() * (double)(glen - frag + 1));
      const bool minus = r.uniform() < 0.5;
      const uint8_t* fwd = genome + start;
      const uint8_t* end = genome + start + frag - read_len;
      // end read on the reverse strand: complement of the end, reversed
      for (uint32_t j = 0; j < read_len; j++) {
        const uint8_t a1 = fwd[j], a2 = (uint8_t)(3 - end[read_len - 1 - j]);
        r1[j] = minus ? a2 : a1;
        r2[j] = minus ? a1 : a2;
      }
      for (int m = 0; m < 2; m++) {
        std::vector<uint8_t>& rr = m ? r2 : r1;
        for (uint32_t j = 0; j < read_len; j++)
          if (r.uniform() < err) rr[j] = (uint8_t)((rr[j] + 1 + (r.next() % 3)) & 3);
        const uint64_t idx = (m ? first2 : first1) + i;
        uint8_t* p = data + idx * nb;
        std::memset(p, 0, nb);
        for (uint32_t j = 0; j < read_len; j++) p[j >> 2] |= (uint8_t)(rr[j] << (6 - 2 * (j & 3)));
        offsets[idx] = idx * nb;
        lengths[idx] = read_len;
      }
    }
  });
}

}  // extern "C"
