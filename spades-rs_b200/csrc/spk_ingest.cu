// spk_ingest.cu -- FASTQ / FASTA text to the PackedReads store on the device:
// FastxReader (src/packed_reads.rs:69-234) and the three-gate, three-block
// ingest of from_paired_files / append_from_file (:300-381, :493-504,
// :513-578, :635-690).  Gzip stays with the caller: the texts arrive
// decompressed.
//
// Per text: newline positions (chunk counts, scan, ordered write) -> line
// bounds -> record structure (FASTQ: a parallel scan over the per-line
// transition functions of the reader's 4-state record machine; FASTA: header
// lines) -> the sequence lines copied into one compact buffer -> per record,
// one warp finds its runs of A/C/G/T bytes.  The runs decide everything the
// gates need: the terminal trim is the span from the first run's start to the
// last run's end, an internal N exists iff there are two runs or more, and the
// sub-reads of the N split are the runs of at least MIN_K bases.  A plan per
// unit (a pair of records, or one record without a mate) then gives every
// packed read its index and byte offset in Block 1 (clean R1), Block 2 (clean
// R2) or Block 3 (split and unpaired reads), and a final pass packs them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "spk_internal.h"

namespace spk {

constexpr int kIgBlock = 256;
constexpr uint32_t kIgChunk = 4096;  // text bytes per CTA in the newline passes
constexpr uint32_t kMinK = 21;       // MIN_K, src/packed_reads.rs:38

// Error codes; the device error word holds (first failing line << 8) | code.
enum IgErr : uint32_t {
  IG_OK = 0,
  IG_HEADER = 1,   // FASTQ: a record does not start with '@'
  IG_PLUS = 3,     // FASTQ: the third line does not start with '+'
  IG_QUAL = 4,     // FASTQ: quality length != sequence length
};

__device__ __forceinline__ int ig_code(uint8_t c) {
  switch (c | 0x20) {  // base_to_2bit, src/dna.rs:30-37 (either case)
    case 'a': return 0;
    case 'c': return 1;
    case 'g': return 2;
    case 't': return 3;
    default: return -1;
  }
}

// ---- newlines ---------------------------------------------------------------
__global__ void __launch_bounds__(kIgBlock) k_ig_nl_count(const uint8_t* __restrict__ t, uint64_t n,
                                                          uint32_t* __restrict__ cnt) {
  __shared__ uint32_t ws[kIgBlock / 32];
  const uint64_t c0 = (uint64_t)blockIdx.x * kIgChunk;
  uint32_t c = 0;
  for (uint32_t j = threadIdx.x; j < kIgChunk; j += kIgBlock) {
    const uint64_t i = c0 + j;
    c += (i < n && t[i] == '\n') ? 1u : 0u;
  }
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int w = 0; w < kIgBlock / 32; w++) s += ws[w];
    cnt[blockIdx.x] = s;
  }
}
// Newline positions in text order; base[chunk] = newlines before the chunk.
__global__ void __launch_bounds__(kIgBlock) k_ig_nl_write(const uint8_t* __restrict__ t, uint64_t n,
                                                          const uint32_t* __restrict__ base,
                                                          uint32_t* __restrict__ nlpos) {
  __shared__ uint32_t ws[kIgBlock / 32];
  const uint64_t c0 = (uint64_t)blockIdx.x * kIgChunk;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t run = base[blockIdx.x];
  // rounds of kIgBlock consecutive bytes, in order
  for (uint32_t j0 = 0; j0 < kIgChunk; j0 += kIgBlock) {
    const uint64_t i = c0 + j0 + threadIdx.x;
    const bool nl = i < n && t[i] == '\n';
    const uint32_t m = __ballot_sync(0xffffffffu, nl);
    if (lane == 0) ws[warp] = __popc(m);
    __syncthreads();
    uint32_t before = run;
    for (unsigned w = 0; w < warp; w++) before += ws[w];
    uint32_t total = 0;
    for (unsigned w = 0; w < kIgBlock / 32; w++) total += ws[w];
    if (nl) nlpos[before + __popc(m & ((1u << lane) - 1u))] = (uint32_t)i;
    run += total;
    __syncthreads();
  }
}

// ---- lines ------------------------------------------------------------------
// Line i: raw bytes [start, end) without its '\n'; content = [start, cend)
// after the trailing '\r' bytes are dropped (next_seq pops '\n' and '\r').
struct IgLines {
  const uint32_t* nlpos;  // newline positions
  uint32_t n_nl;
  uint32_t n_lines;       // n_nl, plus one for text after the last newline
  uint64_t n;             // text bytes
};
__device__ __forceinline__ void ig_line(const IgLines& L, const uint8_t* t, uint32_t i, uint32_t* s,
                                        uint32_t* e, uint32_t* ce) {
  *s = i ? L.nlpos[i - 1] + 1u : 0u;
  *e = i < L.n_nl ? L.nlpos[i] : (uint32_t)L.n;
  uint32_t c = *e;
  while (c > *s && t[c - 1] == '\r') c--;
  *ce = c;
}

// FASTQ record machine (src/packed_reads.rs:146-212): states H (header
// expected; blank lines skipped), S (sequence), P ('+' line), Q (quality).
// A line maps the state before it to the state after it; as a function it
// is 4 x 2 bits, f(s) = (f >> 2s) & 3.  Non-blank: H->S, S->P, P->Q, Q->H;
// blank: H->H, the rest as non-blank.
constexpr uint8_t kFsmNonBlank = 1 | (2 << 2) | (3 << 4) | (0 << 6);
constexpr uint8_t kFsmBlank = 0 | (2 << 2) | (3 << 4) | (0 << 6);
__device__ __forceinline__ uint32_t fsm_then(uint32_t f, uint32_t g) {  // g after f
  uint32_t h = 0;
#pragma unroll
  for (int s = 0; s < 4; s++) h |= ((g >> (2 * ((f >> (2 * s)) & 3))) & 3) << (2 * s);
  return h;
}
constexpr uint32_t kFsmId = 0 | (1 << 2) | (2 << 4) | (3 << 6);

// Block-local exclusive scan of the line functions; agg[block] = the block's
// composite.
__global__ void __launch_bounds__(1024) k_ig_fsm_local(IgLines L, const uint8_t* __restrict__ t,
                                                       uint8_t* __restrict__ pre, uint8_t* __restrict__ agg) {
  __shared__ uint32_t ws[32];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
  uint32_t f = kFsmId;
  if (i < L.n_lines) {
    uint32_t s, e, ce;
    ig_line(L, t, i, &s, &e, &ce);
    f = ce > s ? kFsmNonBlank : kFsmBlank;
  }
  uint32_t x = f;  // inclusive composite of lanes 0..lane
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if ((int)lane >= d) x = fsm_then(y, x);
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t z = ws[lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, z, d);
      if ((int)lane >= d) z = fsm_then(y, z);
    }
    ws[lane] = z;  // inclusive over warps 0..lane
  }
  __syncthreads();
  const uint32_t wpre = warp ? ws[warp - 1] : kFsmId;
  uint32_t lpre = __shfl_up_sync(0xffffffffu, x, 1);
  if (lane == 0) lpre = kFsmId;
  if (i < L.n_lines) pre[i] = (uint8_t)fsm_then(wpre, lpre);
  if (threadIdx.x == 0) agg[blockIdx.x] = (uint8_t)ws[31];
}
// Exclusive scan of the block composites (one CTA, sequential over chunks).
__global__ void __launch_bounds__(1024) k_ig_fsm_blocks(uint8_t* __restrict__ agg, uint32_t nb,
                                                        uint8_t* __restrict__ final_state) {
  __shared__ uint32_t ws[32];
  __shared__ uint32_t carry;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = kFsmId;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < nb; b0 += 1024) {
    const uint32_t i = b0 + threadIdx.x;
    const uint32_t f = i < nb ? agg[i] : kFsmId;
    uint32_t x = f;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if ((int)lane >= d) x = fsm_then(y, x);
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t z = ws[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, z, d);
        if ((int)lane >= d) z = fsm_then(y, z);
      }
      ws[lane] = z;
    }
    __syncthreads();
    const uint32_t c = carry;
    const uint32_t wpre = warp ? ws[warp - 1] : kFsmId;
    uint32_t lpre = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) lpre = kFsmId;
    if (i < nb) agg[i] = (uint8_t)fsm_then(c, fsm_then(wpre, lpre));
    __syncthreads();
    if (threadIdx.x == 0) carry = fsm_then(c, ws[31]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *final_state = (uint8_t)(carry & 3);  // state after the last line, from H
}

// Per line (FASTQ): the state before it, the checks, and the sequence bytes
// it contributes; rec[i] = 1 for a record's sequence line.
__global__ void __launch_bounds__(kIgBlock) k_ig_fastq_lines(IgLines L, const uint8_t* __restrict__ t,
                                                             const uint8_t* __restrict__ pre,
                                                             const uint8_t* __restrict__ agg,
                                                             uint32_t* __restrict__ seqlen,
                                                             uint32_t* __restrict__ rec,
                                                             unsigned long long* __restrict__ err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n_lines; i += gridDim.x * blockDim.x) {
    const uint32_t st = fsm_then(agg[i >> 10], pre[i]) & 3;  // from H
    uint32_t s, e, ce;
    ig_line(L, t, i, &s, &e, &ce);
    uint32_t code = IG_OK;
    uint32_t sl = 0, r = 0;
    if (st == 0) {
      if (ce > s && t[s] != '@') code = IG_HEADER;
    } else if (st == 1) {
      sl = ce - s;
      r = 1;
    } else if (st == 2) {
      if (!(e > s && t[s] == '+')) code = IG_PLUS;  // the raw line starts with '+'
    } else if (i >= 2) {
      uint32_t ps, pe_, pce;
      ig_line(L, t, i - 2, &ps, &pe_, &pce);  // the sequence line of this record
      if (ce - s != pce - ps) code = IG_QUAL;
    } else {
      code = IG_QUAL;  // unreachable: Q follows S and P
    }
    seqlen[i] = sl;
    rec[i] = r;
    if (code) atomicMin(err, ((unsigned long long)i << 8) | code);
  }
}

// Per line (FASTA, src/packed_reads.rs:214-231): header lines start records
// and contribute no bytes; every other line contributes its content.
__global__ void __launch_bounds__(kIgBlock) k_ig_fasta_lines(IgLines L, const uint8_t* __restrict__ t,
                                                             uint32_t* __restrict__ seqlen,
                                                             uint32_t* __restrict__ rec) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n_lines; i += gridDim.x * blockDim.x) {
    uint32_t s, e, ce;
    ig_line(L, t, i, &s, &e, &ce);
    const bool hdr = ce > s && t[s] == '>';
    seqlen[i] = hdr ? 0u : ce - s;
    rec[i] = hdr ? 1u : 0u;
  }
}

// Sequence lines copied to the compact buffer (one warp per line);
// rec_start[r] = the first byte of record r there.
__global__ void __launch_bounds__(kIgBlock) k_ig_copy(IgLines L, const uint8_t* __restrict__ t,
                                                      const uint32_t* __restrict__ seqpos,
                                                      const uint32_t* __restrict__ recidx, int fastq,
                                                      uint8_t* __restrict__ seq, uint32_t* __restrict__ rec_start,
                                                      uint32_t* __restrict__ rec_len) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x / 32);
  for (uint32_t i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); i < L.n_lines; i += nw) {
    uint32_t s, e, ce;
    ig_line(L, t, i, &s, &e, &ce);
    const bool isrec = recidx[i + 1] != recidx[i];
    const bool hdr = !fastq && isrec;
    if (isrec && lane == 0) {
      rec_start[recidx[i]] = seqpos[i];
      if (fastq) rec_len[recidx[i]] = ce - s;
    }
    const bool content = fastq ? isrec : !hdr;
    if (!content) continue;
    const uint32_t o = seqpos[i];
    for (uint32_t j = lane; j < ce - s; j += 32) seq[o + j] = t[s + j];
  }
}
__global__ void k_ig_fasta_len(const uint32_t* __restrict__ rec_start, uint32_t nrec, uint32_t total,
                               uint32_t* __restrict__ rec_len) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += gridDim.x * blockDim.x)
    rec_len[r] = (r + 1 < nrec ? rec_start[r + 1] : total) - rec_start[r];
}

// ---- records ------------------------------------------------------------------
// Runs of A/C/G/T bytes of each record.  Per record: the number of runs, the
// first run's start and the last run's end (the terminal trim,
// src/packed_reads.rs:635-648), and the runs of at least MIN_K bases (the
// N split of :521-540, :659-662): their number and packed bytes.
struct IgRec {
  uint32_t nruns, a, b, nseg, segbytes, pad;
};
// Calls emit(start, len) in order for every run of the record (all lanes).
template <class F>
__device__ __forceinline__ void ig_runs(const uint8_t* seq, uint32_t len, unsigned lane, F emit) {
  uint32_t run = 0, rs = 0;
  for (uint32_t c0 = 0; c0 < len; c0 += 32) {
    const uint32_t j = c0 + lane;
    const bool ok = j < len && ig_code(seq[j]) >= 0;
    const uint32_t m = __ballot_sync(0xffffffffu, ok);
    const uint32_t nv = min(32u, len - c0);
    uint32_t p = 0;
    while (p < nv) {
      const uint32_t mm = m >> p;  // p < 32
      if (mm & 1u) {
        const uint32_t ones = (~mm) ? (uint32_t)(__ffs(~mm) - 1) : 32u - p;
        const uint32_t r = min(ones, nv - p);
        if (run == 0) rs = c0 + p;
        run += r;
        p += r;
      } else {
        if (run) emit(rs, run);
        run = 0;
        const uint32_t z = mm ? (uint32_t)(__ffs(mm) - 1) : nv - p;
        p += min(z, nv - p);
      }
    }
  }
  if (run) emit(rs, run);
}
__global__ void __launch_bounds__(kIgBlock) k_ig_records(const uint8_t* __restrict__ seq,
                                                         const uint32_t* __restrict__ rec_start,
                                                         const uint32_t* __restrict__ rec_len, uint32_t nrec,
                                                         IgRec* __restrict__ out) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x / 32);
  for (uint32_t r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); r < nrec; r += nw) {
    IgRec q{0, 0, 0, 0, 0, 0};
    ig_runs(seq + rec_start[r], rec_len[r], lane, [&](uint32_t s, uint32_t len) {
      if (q.nruns == 0) q.a = s;
      q.nruns++;
      q.b = s + len;
      if (len >= kMinK) {
        q.nseg++;
        q.segbytes += (len + 3) / 4;
      }
    });
    if (lane == 0) out[r] = q;
  }
}

// ---- plan ------------------------------------------------------------------------
// Units: u < common pairs record u of both texts (partition_pair_streaming,
// src/packed_reads.rs:668-690); then the records of the longer text without a
// mate, one each (ingest_read, :513-517).  A single text has only the latter.
struct IgPlan {
  uint32_t* c1;      // clean pair: 1 (Block 1 and Block 2 read)
  uint32_t* b1;      // Block 1 bytes (R1)
  uint32_t* b2;      // Block 2 bytes (R2)
  uint32_t* r3;      // Block 3 reads
  uint32_t* b3;      // Block 3 bytes
  uint32_t* sc;      // sidecar entries
  uint32_t* scb;     // sidecar bytes
};
__device__ __forceinline__ bool ig_clean(const IgRec& q) {  // one run (no internal N) of >= MIN_K
  return q.nruns == 1 && q.b - q.a >= kMinK;
}
__global__ void k_ig_plan(const IgRec* __restrict__ A, uint32_t na, const IgRec* __restrict__ B, uint32_t nb,
                          uint32_t common, uint32_t nunits, IgPlan P) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < nunits; u += gridDim.x * blockDim.x) {
    uint32_t c1 = 0, b1 = 0, b2 = 0, r3 = 0, b3 = 0, sc = 0, scb = 0;
    auto block3 = [&](const IgRec& q) {  // ingest_trimmed_unpaired, :521-540
      r3 += q.nseg;
      b3 += q.segbytes;
      if (q.nruns > 0 && q.nseg == 0) {
        sc++;
        scb += q.b - q.a;
      }
    };
    if (u < common) {
      const IgRec qa = A[u], qb = B[u];
      if (ig_clean(qa) && ig_clean(qb)) {
        c1 = 1;
        b1 = (qa.b - qa.a + 3) / 4;
        b2 = (qb.b - qb.a + 3) / 4;
      } else {
        block3(qa);
        block3(qb);
      }
    } else {
      const uint32_t i = u;  // a record of the longer text
      block3(na > nb ? A[i] : B[i]);
    }
    P.c1[u] = c1;
    P.b1[u] = b1;
    P.b2[u] = b2;
    P.r3[u] = r3;
    P.b3[u] = b3;
    P.sc[u] = sc;
    P.scb[u] = scb;
  }
}

// Packs seq[0, len) (A/C/G/T bytes) to (len + 3) / 4 bytes at out, first base
// in the top bits (pack_clean, src/packed_reads.rs:547-578); one warp.
__device__ __forceinline__ void ig_pack(const uint8_t* seq, uint32_t len, uint8_t* out, unsigned lane) {
  const uint32_t nb = (len + 3) / 4;
  for (uint32_t j = lane; j < nb; j += 32) {
    uint32_t byte = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint32_t p = 4 * j + q;
      if (p < len) byte |= (uint32_t)ig_code(seq[p]) << (6 - 2 * q);
    }
    out[j] = (uint8_t)byte;
  }
}

struct IgText {
  const uint8_t* seq;
  const uint32_t* start;
  const uint32_t* len;
  const IgRec* rec;
  uint32_t nrec;
};
struct IgOut {
  uint8_t* data;
  uint64_t* offsets;
  uint32_t* lengths;
  uint8_t* sidecar;
  uint32_t* sc_len;
  uint32_t pe;            // clean pairs
  uint32_t b1_total;      // bytes of Block 1
  uint32_t b2_total;      // bytes of Block 2
};
// Exclusive scans of the plan arrays give every unit its positions.
__global__ void __launch_bounds__(kIgBlock) k_ig_emit(IgText TA, IgText TB, uint32_t common, uint32_t nunits,
                                                      IgPlan P, IgOut O) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x / 32);
  for (uint32_t u = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); u < nunits; u += nw) {
    const bool pair = u < common;
    const bool clean = pair && P.c1[u + 1] != P.c1[u];
    if (clean) {
      const uint32_t idx = P.c1[u];
      const IgRec qa = TA.rec[u], qb = TB.rec[u];
      const uint32_t la = qa.b - qa.a, lb = qb.b - qb.a;
      const uint32_t oa = P.b1[u], ob = O.b1_total + P.b2[u];
      ig_pack(TA.seq + TA.start[u] + qa.a, la, O.data + oa, lane);
      ig_pack(TB.seq + TB.start[u] + qb.a, lb, O.data + ob, lane);
      if (lane == 0) {
        O.offsets[idx] = oa;
        O.lengths[idx] = la;
        O.offsets[O.pe + idx] = ob;
        O.lengths[O.pe + idx] = lb;
      }
      continue;
    }
    uint32_t ridx = 2 * O.pe + P.r3[u];
    uint32_t boff = O.b1_total + O.b2_total + P.b3[u];
    uint32_t sidx = P.sc[u], soff = P.scb[u];
    auto block3 = [&](const IgText& T, uint32_t r) {
      const uint8_t* s = T.seq + T.start[r];
      const IgRec q = T.rec[r];
      ig_runs(s, T.len[r], lane, [&](uint32_t rs, uint32_t rl) {
        if (rl < kMinK) return;
        ig_pack(s + rs, rl, O.data + boff, lane);
        if (lane == 0) {
          O.offsets[ridx] = boff;
          O.lengths[ridx] = rl;
        }
        ridx++;
        boff += (rl + 3) / 4;
      });
      if (q.nruns > 0 && q.nseg == 0) {  // Gate 3: the trimmed read goes to the sidecar
        for (uint32_t j = lane; j < q.b - q.a; j += 32) O.sidecar[soff + j] = s[q.a + j];
        if (lane == 0) O.sc_len[sidx] = q.b - q.a;
        sidx++;
        soff += q.b - q.a;
      }
    };
    if (pair) {
      block3(TA, u);
      block3(TB, u);
    } else if (TA.nrec > TB.nrec) {
      block3(TA, u);
    } else {
      block3(TB, u);
    }
  }
}

// ---- host ------------------------------------------------------------------------
struct TextDev {
  DevBuf text, nl, seqlen, rec, seq, start, len, recs;
  uint32_t nrec = 0;
  uint32_t total = 0;  // compact sequence bytes
};

static std::string ig_message(uint32_t code) {
  switch (code) {
    case IG_HEADER: return "Malformed FASTQ record: expected '@' header";
    case IG_PLUS: return "Malformed FASTQ record: expected '+' separator line";
    case IG_QUAL: return "Malformed FASTQ record: sequence length != quality length";
    default: return "Malformed FASTQ record";
  }
}

// FastxReader::open (src/packed_reads.rs:69-135): leading blank or
// whitespace-only lines are skipped; the first byte then picks the format.
// Returns the offset of the first record (after the first '>' header line
// for FASTA); *fmt = 1 FASTQ, 0 FASTA, -1 empty.
static int ig_open(const uint8_t* t, uint64_t n, uint64_t* off, int* fmt) {
  uint64_t p = 0;
  for (;;) {
    if (p >= n) {
      *fmt = -1;
      *off = n;
      return SPK_OK;
    }
    uint64_t e = p;
    while (e < n && t[e] != '\n') e++;
    bool ws = true;
    for (uint64_t i = p; i < e && ws; i++)
      ws = t[i] == ' ' || t[i] == '\t' || t[i] == '\r' || t[i] == '\x0c';
    if (!ws) break;
    p = e < n ? e + 1 : e;
  }
  if (t[p] == '@') {
    *fmt = 1;
    *off = p;
    return SPK_OK;
  }
  if (t[p] != '>') return fail(SPK_E_INVALID_ARG, "Malformed FASTQ/FASTA file: expected '@' or '>' header");
  uint64_t e = p;
  while (e < n && t[e] != '\n') e++;
  *fmt = 0;
  *off = e < n ? e + 1 : e;
  return SPK_OK;
}

static unsigned ig_grid(spk_ctx* ctx, uint64_t items, unsigned per_block) {
  const uint64_t want = (items + per_block - 1) / per_block;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)ctx->sm_count * 16));
}

// One text to records on the device.
static int ig_text(spk_ctx* ctx, cudaStream_t st, const uint8_t* host, uint64_t n_all, TextDev& T,
                   uint32_t* launches) {
  uint64_t off = 0;
  int fmt = -1, rc;
  if ((rc = ig_open(host, n_all, &off, &fmt))) return rc;
  if (fmt < 0) return SPK_OK;
  const uint64_t n = n_all - off;
  if (n >= 0xFFFFFFF0ull) return fail(SPK_E_INVALID_ARG, "a FASTQ/FASTA text of 4 GiB or more");
  if ((rc = T.text.alloc(n + 64, st))) return rc;
  SPK_CUDA(cudaMemcpyAsync(T.text.p, host + off, n, cudaMemcpyHostToDevice, st));
  const uint8_t* t = T.text.as<uint8_t>();
  DevBuf cnt, sums, err;
  const uint32_t nchunks = (uint32_t)((n + kIgChunk - 1) / kIgChunk);
  if ((rc = cnt.alloc((uint64_t)(nchunks + 1) * 4, st)) || (rc = err.alloc(8, st))) return rc;
  SPK_CUDA(cudaMemsetAsync(cnt.p, 0, (uint64_t)(nchunks + 1) * 4, st));
  SPK_CUDA(cudaMemsetAsync(err.p, 0xFF, 8, st));
  if (nchunks) k_ig_nl_count<<<nchunks, kIgBlock, 0, st>>>(t, n, cnt.as<uint32_t>());
  if ((rc = scan_u32(st, cnt.as<uint32_t>(), (uint64_t)nchunks + 1, sums, launches))) return rc;
  uint32_t n_nl = 0;
  SPK_CUDA(cudaMemcpyAsync(&n_nl, cnt.as<uint32_t>() + nchunks, 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  if ((rc = T.nl.alloc((uint64_t)n_nl * 4 + 4, st))) return rc;
  if (nchunks) k_ig_nl_write<<<nchunks, kIgBlock, 0, st>>>(t, n, cnt.as<uint32_t>(), T.nl.as<uint32_t>());
  uint32_t last_nl = 0;
  if (n_nl) {
    SPK_CUDA(cudaMemcpyAsync(&last_nl, T.nl.as<uint32_t>() + n_nl - 1, 4, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
  }
  const bool tail = n_nl ? (uint64_t)last_nl + 1 < n : n > 0;
  IgLines L{T.nl.as<uint32_t>(), n_nl, n_nl + (tail ? 1u : 0u), n};
  if (launches) *launches += 2;
  if (L.n_lines == 0) return SPK_OK;
  if ((rc = T.seqlen.alloc((uint64_t)L.n_lines * 4 + 4, st)) || (rc = T.rec.alloc((uint64_t)L.n_lines * 4 + 4, st)))
    return rc;
  SPK_CUDA(cudaMemsetAsync(T.seqlen.as<uint32_t>() + L.n_lines, 0, 4, st));
  SPK_CUDA(cudaMemsetAsync(T.rec.as<uint32_t>() + L.n_lines, 0, 4, st));
  const unsigned g = ig_grid(ctx, L.n_lines, kIgBlock);
  uint32_t final_state = 0;
  if (fmt == 1) {
    const uint32_t nb = (L.n_lines + 1023) / 1024;
    DevBuf pre, agg, fin;
    if ((rc = pre.alloc(L.n_lines, st)) || (rc = agg.alloc(nb, st)) || (rc = fin.alloc(4, st))) return rc;
    k_ig_fsm_local<<<nb, 1024, 0, st>>>(L, t, pre.as<uint8_t>(), agg.as<uint8_t>());
    k_ig_fsm_blocks<<<1, 1024, 0, st>>>(agg.as<uint8_t>(), nb, fin.as<uint8_t>());
    k_ig_fastq_lines<<<g, kIgBlock, 0, st>>>(L, t, pre.as<uint8_t>(), agg.as<uint8_t>(), T.seqlen.as<uint32_t>(),
                                             T.rec.as<uint32_t>(), err.as<unsigned long long>());
    uint8_t fs = 0;
    SPK_CUDA(cudaMemcpyAsync(&fs, fin.p, 1, cudaMemcpyDeviceToHost, st));
    unsigned long long he = 0;
    SPK_CUDA(cudaMemcpyAsync(&he, err.p, 8, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    if (launches) *launches += 3;
    if (he != ~0ull)
      return fail(SPK_E_INVALID_ARG, ig_message((uint32_t)(he & 0xFF)) + " (line " + std::to_string(he >> 8) +
                                         " after the leading blank lines)");
    final_state = fs;
    if (final_state == 1) return fail(SPK_E_INVALID_ARG, "Malformed FASTQ record: unexpected EOF waiting for sequence line");
    if (final_state == 2) return fail(SPK_E_INVALID_ARG, "Malformed FASTQ record: unexpected EOF waiting for '+' separator");
    if (final_state == 3) return fail(SPK_E_INVALID_ARG, "Malformed FASTQ record: unexpected EOF waiting for quality scores");
  } else {
    // FASTA: the text starts after the first header; record 0 begins at line
    // 0 as if a header preceded it.  The flag array marks header lines, so
    // add the implicit first record by hand after the scan.
    k_ig_fasta_lines<<<g, kIgBlock, 0, st>>>(L, t, T.seqlen.as<uint32_t>(), T.rec.as<uint32_t>());
    if (launches) *launches += 1;
  }
  // positions of sequence bytes and record indices
  DevBuf seqpos, recidx;
  if ((rc = seqpos.alloc((uint64_t)L.n_lines * 4 + 4, st)) || (rc = recidx.alloc((uint64_t)L.n_lines * 4 + 8, st)))
    return rc;
  SPK_CUDA(cudaMemcpyAsync(seqpos.p, T.seqlen.p, (uint64_t)L.n_lines * 4 + 4, cudaMemcpyDeviceToDevice, st));
  SPK_CUDA(cudaMemcpyAsync(recidx.p, T.rec.p, (uint64_t)L.n_lines * 4 + 4, cudaMemcpyDeviceToDevice, st));
  if ((rc = scan_u32(st, seqpos.as<uint32_t>(), (uint64_t)L.n_lines + 1, sums, launches))) return rc;
  if ((rc = scan_u32(st, recidx.as<uint32_t>(), (uint64_t)L.n_lines + 1, sums, launches))) return rc;
  uint32_t h2[2];
  SPK_CUDA(cudaMemcpyAsync(&h2[0], seqpos.as<uint32_t>() + L.n_lines, 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaMemcpyAsync(&h2[1], recidx.as<uint32_t>() + L.n_lines, 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  T.total = h2[0];
  uint32_t nrec = h2[1];
  if ((rc = T.seq.alloc((uint64_t)T.total + 64, st))) return rc;
  if (fmt == 1) {
    if ((rc = T.start.alloc((uint64_t)nrec * 4 + 4, st)) || (rc = T.len.alloc((uint64_t)nrec * 4 + 4, st))) return rc;
    if (L.n_lines)
      k_ig_copy<<<g, kIgBlock, 0, st>>>(L, t, seqpos.as<uint32_t>(), recidx.as<uint32_t>(), 1, T.seq.as<uint8_t>(),
                                        T.start.as<uint32_t>(), T.len.as<uint32_t>());
    if (launches) *launches += 1;
  } else {
    // Records: the implicit first one (index 0, starting at byte 0) and one
    // per header line (index recidx + 1).  Shift by writing starts at +1.
    if ((rc = T.start.alloc((uint64_t)nrec * 4 + 8, st)) || (rc = T.len.alloc((uint64_t)nrec * 4 + 8, st))) return rc;
    SPK_CUDA(cudaMemsetAsync(T.start.p, 0, 4, st));
    k_ig_copy<<<g, kIgBlock, 0, st>>>(L, t, seqpos.as<uint32_t>(), recidx.as<uint32_t>(), 0, T.seq.as<uint8_t>(),
                                      T.start.as<uint32_t>() + 1, nullptr);
    nrec += 1;
    k_ig_fasta_len<<<ig_grid(ctx, nrec, kIgBlock), kIgBlock, 0, st>>>(T.start.as<uint32_t>(), nrec, T.total,
                                                                       T.len.as<uint32_t>());
    // next_seq at EOF returns a record only if its sequence is not empty
    uint32_t last_len = 0;
    SPK_CUDA(cudaMemcpyAsync(&last_len, T.len.as<uint32_t>() + nrec - 1, 4, cudaMemcpyDeviceToHost, st));
    SPK_CUDA(cudaStreamSynchronize(st));
    if (last_len == 0) nrec -= 1;
    if (launches) *launches += 2;
  }
  T.nrec = nrec;
  if (nrec) {
    if ((rc = T.recs.alloc((uint64_t)nrec * sizeof(IgRec), st))) return rc;
    k_ig_records<<<ig_grid(ctx, nrec, kIgBlock / 32), kIgBlock, 0, st>>>(T.seq.as<uint8_t>(), T.start.as<uint32_t>(),
                                                                          T.len.as<uint32_t>(), nrec,
                                                                          T.recs.as<IgRec>());
    if (launches) *launches += 1;
  }
  SPK_CUDA(cudaGetLastError());
  T.text.release();
  T.seqlen.release();
  T.rec.release();
  T.nl.release();
  return SPK_OK;
}

}  // namespace spk

using namespace spk;

struct spk_packed {
  spk_ctx* ctx = nullptr;
  spk::DevBuf data, offsets, lengths;
  uint64_t n_reads = 0, data_len = 0, pe_count = 0;
  std::vector<uint8_t> sidecar;          // concatenated trimmed reads
  std::vector<uint64_t> sidecar_len;
  uint32_t launches = 0;
  float ms = 0.f;
};

static int ingest_impl(spk_ctx* ctx, const uint8_t* t1, size_t l1, const uint8_t* t2, size_t l2, bool paired,
                       spk_packed* P) {
  cudaStream_t st = ctx->stream;
  TextDev A, B;
  int rc;
  if ((rc = ig_text(ctx, st, t1, l1, A, &P->launches))) return rc;
  if (paired && (rc = ig_text(ctx, st, t2, l2, B, &P->launches))) return rc;
  const uint32_t na = A.nrec, nb = paired ? B.nrec : 0;
  const uint32_t common = std::min(na, nb);
  const uint32_t nunits = std::max(na, nb);
  DevBuf plan, sums;
  const uint64_t pn = (uint64_t)nunits + 1;
  if ((rc = plan.alloc(pn * 4 * 7, st))) return rc;
  SPK_CUDA(cudaMemsetAsync(plan.p, 0, pn * 4 * 7, st));
  uint32_t* pb = plan.as<uint32_t>();
  IgPlan Pl{pb, pb + pn, pb + 2 * pn, pb + 3 * pn, pb + 4 * pn, pb + 5 * pn, pb + 6 * pn};
  if (nunits) {
    k_ig_plan<<<ig_grid(ctx, nunits, kIgBlock), kIgBlock, 0, st>>>(A.recs.as<IgRec>(), na, B.recs.as<IgRec>(), nb,
                                                                   common, nunits, Pl);
    P->launches++;
  }
  for (int a = 0; a < 7; a++)
    if ((rc = scan_u32(st, pb + a * pn, pn, sums, &P->launches))) return rc;
  uint32_t tot[7];
  for (int a = 0; a < 7; a++)
    SPK_CUDA(cudaMemcpyAsync(&tot[a], pb + a * pn + nunits, 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  const uint64_t pe = tot[0], r3 = tot[3];
  const uint64_t nreads = 2 * pe + r3;
  const uint64_t dlen = (uint64_t)tot[1] + tot[2] + tot[4];
  DevBuf scd, scl;
  if ((rc = P->data.alloc(dlen + 64, st)) || (rc = P->offsets.alloc(std::max<uint64_t>(nreads, 1) * 8, st)) ||
      (rc = P->lengths.alloc(std::max<uint64_t>(nreads, 1) * 4, st)) ||
      (rc = scd.alloc((uint64_t)tot[6] + 1, st)) || (rc = scl.alloc((uint64_t)tot[5] * 4 + 4, st)))
    return rc;
  SPK_CUDA(cudaMemsetAsync(P->data.p, 0, dlen + 64, st));
  if (nunits) {
    IgText TA{A.seq.as<uint8_t>(), A.start.as<uint32_t>(), A.len.as<uint32_t>(), A.recs.as<IgRec>(), na};
    IgText TB{B.seq.as<uint8_t>(), B.start.as<uint32_t>(), B.len.as<uint32_t>(), B.recs.as<IgRec>(), nb};
    IgOut O{P->data.as<uint8_t>(), P->offsets.as<uint64_t>(), P->lengths.as<uint32_t>(), scd.as<uint8_t>(),
            scl.as<uint32_t>(), (uint32_t)pe, tot[1], tot[2]};
    k_ig_emit<<<ig_grid(ctx, nunits, kIgBlock / 32), kIgBlock, 0, st>>>(TA, TB, common, nunits, Pl, O);
    SPK_CUDA(cudaGetLastError());
    P->launches++;
  }
  P->sidecar.resize(tot[6]);
  std::vector<uint32_t> sl(tot[5]);
  if (tot[6]) SPK_CUDA(cudaMemcpyAsync(P->sidecar.data(), scd.p, tot[6], cudaMemcpyDeviceToHost, st));
  if (tot[5]) SPK_CUDA(cudaMemcpyAsync(sl.data(), scl.p, (uint64_t)tot[5] * 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  P->sidecar_len.assign(sl.begin(), sl.end());
  P->n_reads = nreads;
  P->data_len = dlen;
  P->pe_count = pe;
  return SPK_OK;
}

extern "C" int spk_ingest(spk_ctx* ctx, const uint8_t* text1, size_t len1, const uint8_t* text2, size_t len2,
                          spk_packed** out) {
  if (!ctx || !out) return fail(SPK_E_INVALID_ARG, "null argument");
  if ((len1 && !text1) || (len2 && !text2)) return fail(SPK_E_INVALID_ARG, "null text");
  SPK_CUDA(cudaSetDevice(ctx->device));
  auto* P = new spk_packed();
  P->ctx = ctx;
  cudaEvent_t e0, e1;
  SPK_CUDA(cudaEventCreate(&e0));
  SPK_CUDA(cudaEventCreate(&e1));
  cudaEventRecord(e0, ctx->stream);
  int rc = ingest_impl(ctx, text1, len1, text2, len2, text2 != nullptr, P);
  if (!rc) {
    cudaEventRecord(e1, ctx->stream);
    if (cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&P->ms, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    delete P;
    return rc;
  }
  *out = P;
  return SPK_OK;
}

extern "C" int spk_packed_info(const spk_packed* p, uint64_t* n_reads, uint64_t* data_len, uint64_t* pe_count,
                               uint64_t* n_sidecar, uint64_t* sidecar_bytes) {
  if (!p) return fail(SPK_E_INVALID_ARG, "null packed reads");
  if (n_reads) *n_reads = p->n_reads;
  if (data_len) *data_len = p->data_len;
  if (pe_count) *pe_count = p->pe_count;
  if (n_sidecar) *n_sidecar = p->sidecar_len.size();
  if (sidecar_bytes) *sidecar_bytes = p->sidecar.size();
  return SPK_OK;
}

extern "C" int spk_packed_stats(const spk_packed* p, float* ms_device, uint32_t* kernel_launches) {
  if (!p) return fail(SPK_E_INVALID_ARG, "null packed reads");
  if (ms_device) *ms_device = p->ms;
  if (kernel_launches) *kernel_launches = p->launches;
  return SPK_OK;
}

extern "C" int spk_packed_download(spk_packed* p, uint8_t* data, uint64_t* offsets, uint32_t* lengths,
                                   uint8_t* sidecar, uint64_t* sidecar_lengths) {
  if (!p) return fail(SPK_E_INVALID_ARG, "null packed reads");
  SPK_CUDA(cudaSetDevice(p->ctx->device));
  cudaStream_t st = p->ctx->stream;
  if (data && p->data_len) SPK_CUDA(cudaMemcpyAsync(data, p->data.p, p->data_len, cudaMemcpyDeviceToHost, st));
  if (offsets && p->n_reads)
    SPK_CUDA(cudaMemcpyAsync(offsets, p->offsets.p, p->n_reads * 8, cudaMemcpyDeviceToHost, st));
  if (lengths && p->n_reads)
    SPK_CUDA(cudaMemcpyAsync(lengths, p->lengths.p, p->n_reads * 4, cudaMemcpyDeviceToHost, st));
  SPK_CUDA(cudaStreamSynchronize(st));
  if (sidecar && !p->sidecar.empty()) memcpy(sidecar, p->sidecar.data(), p->sidecar.size());
  if (sidecar_lengths && !p->sidecar_len.empty())
    memcpy(sidecar_lengths, p->sidecar_len.data(), p->sidecar_len.size() * 8);
  return SPK_OK;
}

extern "C" int spk_packed_device(spk_packed* p, const uint8_t** d_data, const uint64_t** d_offsets,
                                 const uint32_t** d_lengths) {
  if (!p) return fail(SPK_E_INVALID_ARG, "null packed reads");
  if (d_data) *d_data = p->data.as<uint8_t>();
  if (d_offsets) *d_offsets = p->offsets.as<uint64_t>();
  if (d_lengths) *d_lengths = p->lengths.as<uint32_t>();
  return SPK_OK;
}

extern "C" int spk_packed_free(spk_packed* p) {
  if (!p) return SPK_OK;
  if (p->ctx) cudaSetDevice(p->ctx->device);
  delete p;
  return SPK_OK;
}
