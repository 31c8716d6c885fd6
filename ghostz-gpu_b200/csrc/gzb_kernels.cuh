// gzb_kernels.cuh -- device kernels of the presearch engine (sm_100a).
//
// All arithmetic is int32 and reproduces the CPU reference bit for bit:
//   * ungapped X-drop  : UngappedExtender::ExtendOneSideScoreOnly
//                        (src/ungapped_extender.h:34-82)
//   * distance         : DistanceCalculator::CalculateDistance
//                        (src/distance_calculator.cpp:35-54)
//   * gapped X-drop    : GappedExtender::ExtendOneSideScoreOnly
//                        (src/gapped_extender.cpp:306-471)
//
// Gapped extension, one warp per extension.  The reference walks database
// rows in order and, inside a row, evaluates query columns left to right,
// pruning a cell when the running maximum minus its score exceeds the X-drop
// and resetting the horizontal-gap chain at pruned cells.  The warp evaluates
// 32 consecutive columns of a row at once and stays exact:
//   - a pruned cell's score is always below the running maximum, so the
//     running maximum before a cell equals the plain prefix maximum of the raw
//     scores of the row (one warp max-scan);
//   - without the reset, the horizontal gap F obeys
//     F[c+1] = max(G[c] - gap_init, F[c] - gap_ext)  (G = max(diag, vertical)),
//     a max-plus prefix scan.  Any value the reset would have removed is
//     below (running max - X-drop), so it can neither keep a cell alive nor
//     grow the band; decisions and stored values are unchanged as long as
//     the initial score -1024 itself lies below every live threshold, i.e.
//     X-drop < 1024.  X-drops of at least 2^30 can prune nothing and are
//     exact as well.  Any other X-drop runs the serial fallback.
//   - band edges (array_start / array_end / the sentinel column) follow the
//     reference's rules, including its use of the old right edge when the
//     band shrinks (src/gapped_extender.cpp:449-465).
// The band lives in a per-warp circular buffer of W columns in shared
// memory; an extension whose band would outgrow it is handed to the
// fallback kernel, which keeps the band in a global circular buffer.
#pragma once

#include <cooperative_groups.h>
#include <cstdint>
#include <cuda_runtime.h>

namespace gzb {

namespace cg = cooperative_groups;

constexpr int kInitScore = -(1 << 10);  // src/gapped_extender.h:40
constexpr int kNegBig = -(1 << 29);
// shared-memory score matrix row: 33 words, so that lanes reading different
// rows (their own database residues) at the same column (query residue) hit
// different banks
constexpr int kMatrixStride = 33;

__device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

// Loads a score matrix with row stride `stride` into the shared tile
// (kMatrixStride x kMatrixStride, entries past number_letters zero).
__device__ __forceinline__ void load_matrix(int *sm, const int32_t *m,
                                            int number_letters, int stride) {
  for (int i = threadIdx.x; i < kMatrixStride * kMatrixStride; i += blockDim.x) {
    int r = i / kMatrixStride, c = i % kMatrixStride;
    sm[i] = (r < number_letters && c < number_letters) ? m[r * stride + c] : 0;
  }
}

// ---------------------------------------------------------------------------
// Ungapped one-side X-drop from s0[0]/s1[0] (query/database), stepping by
// INC.  Returns the best prefix sum; stops early once it exceeds stop_above
// (the caller only needs "> trigger").  *steps counts residue pairs
// examined.  Residues are read a 32-bit word at a time (the sequences carry
// readable padding around them), four residue pairs per pair of loads.
template <int INC>
__device__ __forceinline__ int ungapped_side(const uint8_t *__restrict__ s0,
                                             const uint8_t *__restrict__ s1, int delim,
                                             const int *sm, int cutoff, int stop_above,
                                             int *steps) {
  const uint32_t *p0 = (const uint32_t *)((uintptr_t)s0 & ~(uintptr_t)3);
  const uint32_t *p1 = (const uint32_t *)((uintptr_t)s1 & ~(uintptr_t)3);
  int k0 = (int)((uintptr_t)s0 & 3), k1 = (int)((uintptr_t)s1 & 3);
  uint32_t w0 = __ldg(p0), w1 = __ldg(p1);
  int best = 0, run = 0, n = 0;
  for (;;) {
    const int a = (w0 >> (8 * k0)) & 0xff, b = (w1 >> (8 * k1)) & 0xff;
    if (a == delim || b == delim) break;
    run += sm[b * kMatrixStride + a];
    ++n;
    if (INC > 0) {
      if (++k0 == 4) {
        k0 = 0;
        w0 = __ldg(++p0);
      }
      if (++k1 == 4) {
        k1 = 0;
        w1 = __ldg(++p1);
      }
    } else {
      if (--k0 < 0) {
        k0 = 3;
        w0 = __ldg(--p0);
      }
      if (--k1 < 0) {
        k1 = 3;
        w1 = __ldg(--p1);
      }
    }
    if (run > 0) {
      best += run;
      run = 0;
      if (best > stop_above) break;
    } else if (run <= -cutoff) {
      break;
    }
  }
  *steps += n;
  return best;
}

// Ungapped extension with trigger (SeedSearcher::UngappedExtend,
// src/seed_searcher.h:133-158): true when the summed score exceeds trigger.
__device__ __forceinline__ bool ungapped_hit(const uint8_t *q, const uint8_t *d,
                                             int delim, const int *sm,
                                             int cutoff, int trigger,
                                             int *steps) {
  int sum = ungapped_side<-1>(q - 1, d - 1, delim, sm, cutoff, trigger, steps);
  if (sum > trigger) return true;
  sum += ungapped_side<1>(q, d, delim, sm, cutoff, trigger - sum, steps);
  return sum > trigger;
}

// ---------------------------------------------------------------------------
// Ungapped walk over a bank-swizzled score table (the seed-search kernels).
//
// Table layout: the int32 score of (query code a, database code b) sits at
// word (a ^ b) + 64a of an 8 KB shared array (codes < 32), so its bank is
// a ^ b: residue pairs that share a query or a database code land in
// different banks.  The delimiter's row and column hold kWalkDelim, so a
// step onto a delimiter drops the running score by at least 32768 >= cutoff
// and ends the walk with the best score unchanged, exactly as the
// reference's explicit delimiter test does.
constexpr int kWalkTableBytes = 64 * 32 * 4;
constexpr int kWalkDelim = -32768;

__device__ __forceinline__ void load_walk_table(int32_t *tbl, const int32_t *m32, int delim) {
  for (int i = threadIdx.x; i < kWalkTableBytes / 4; i += blockDim.x) {
    const int a = i >> 6, x = i & 63, b = x ^ a;
    int v = 0;
    if (x < 32) v = (a == delim || b == delim) ? kWalkDelim : m32[b * 32 + a];
    tbl[i] = v;
  }
}

template <uint32_t SEL>
__device__ __forceinline__ uint32_t prmt_imm(uint32_t x, uint32_t y) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(y), "n"(SEL));
  return r;
}

// byte offset into the walk table of residue pair j: x4 holds 4(a ^ b) and
// qa holds a in byte j; the result is byte j of x4 | byte j of qa << 8, the
// upper two bytes replicating the (zero) sign bit of byte j of x4
template <int J>
__device__ __forceinline__ uint32_t walk_offset(uint32_t x4, uint32_t qa) {
  return prmt_imm<(uint32_t)(J | ((4 + J) << 4) | ((8 | J) << 8) | ((8 | J) << 12))>(x4, qa);
}

constexpr int kWalkPrefetch = 5;

// One sequence's words around a walk start: chunk k covers residues
// s[4k .. 4k+3] (INC > 0) or s[-4k-3 .. -4k] (INC < 0), and reads the words
// (p[k], p[k + 1]) forward or (p[-k], p[1 - k]) reverse; w[i] holds p[i]
// forward and p[1 - i] reverse for the first kWalkPrefetch chunks.
template <int INC>
struct WalkWords {
  const uint32_t *p;
  uint32_t sh;
  uint32_t w[kWalkPrefetch + 1];
};

template <int INC>
__device__ __forceinline__ void load_walk_words(WalkWords<INC> &ww, const uint8_t *s) {
  const uintptr_t a = (uintptr_t)s - (INC > 0 ? 0 : 3);
  ww.p = (const uint32_t *)(a & ~(uintptr_t)3);
  ww.sh = 8u * (uint32_t)(a & 3);
#pragma unroll
  for (int i = 0; i <= kWalkPrefetch; ++i) ww.w[i] = __ldg(ww.p + (INC > 0 ? i : 1 - i));
}

// walk_side over words already loaded (see walk_side).  A chunk's four
// pairs are scored without an exit test each: the chunk keeps the largest
// drop below the running best (best_j - score_j) and tests it, and the best
// against stop_above, once at its end.  A chunk in which the walk ends is
// then replayed pair by pair from its start (the exact exit pair, its best
// and the step count); no pair after a delimiter changes a value the walk
// returns, since the delimiter's -32768 ends the replay first.
template <int INC>
__device__ __forceinline__ int walk_side_words(const WalkWords<INC> &A, const WalkWords<INC> &B,
                                               const char *tbl, int cutoff, int stop_above,
                                               int *steps) {
  constexpr int K = kWalkPrefetch;
  const uint32_t sha = A.sh, shb = B.sh;
  int score = 0, best = 0, n = 0;
  uint32_t rx4 = 0, rqa = 0;  // the chunk the walk ends in
#define GZB_WALK_V(J, X4, QA) \
  (*(const int32_t *)(tbl + walk_offset<(INC > 0 ? (J) : 3 - (J))>(X4, QA)))
// the four pairs of chunk (X4, QA); leaves the loop for the replay when the
// walk ends inside the chunk
#define GZB_WALK_CHUNK(X4, QA)                                                  \
  {                                                                            \
    const int v0 = GZB_WALK_V(0, X4, QA), v1 = GZB_WALK_V(1, X4, QA);          \
    const int v2 = GZB_WALK_V(2, X4, QA), v3 = GZB_WALK_V(3, X4, QA);          \
    const int s0 = score + v0, b0 = imax(best, s0);                           \
    const int s1 = s0 + v1, b1 = imax(b0, s1);                                \
    const int s2 = s1 + v2, b2 = imax(b1, s2);                                \
    const int s3 = s2 + v3, b3 = imax(b2, s3);                                \
    const int drop = imax(imax(b0 - s0, b1 - s1), imax(b2 - s2, b3 - s3));    \
    if (drop >= cutoff || b3 > stop_above) {                                   \
      rx4 = X4;                                                                \
      rqa = QA;                                                                \
      goto replay;                                                             \
    }                                                                          \
    score = s3;                                                                \
    best = b3;                                                                 \
    n += 4;                                                                    \
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const uint32_t qa = INC > 0 ? __funnelshift_r(A.w[k], A.w[k + 1], sha)
                                : __funnelshift_r(A.w[k + 1], A.w[k], sha);
    const uint32_t qb = INC > 0 ? __funnelshift_r(B.w[k], B.w[k + 1], shb)
                                : __funnelshift_r(B.w[k + 1], B.w[k], shb);
    const uint32_t x4p = (qa ^ qb) << 2;
    GZB_WALK_CHUNK(x4p, qa)
  }
  {
    // past the prefetched chunks: one new word per chunk
    const uint32_t *pa = A.p, *pb = B.p;
    uint32_t a_lo, a_hi, b_lo, b_hi;
    if (INC > 0) {
      pa += K;
      pb += K;
      a_lo = A.w[K];
      b_lo = B.w[K];
      a_hi = __ldg(pa + 1);
      b_hi = __ldg(pb + 1);
    } else {
      pa -= K;
      pb -= K;
      a_hi = A.w[K];
      b_hi = B.w[K];
      a_lo = __ldg(pa);
      b_lo = __ldg(pb);
    }
    for (;;) {
      const uint32_t qa = __funnelshift_r(a_lo, a_hi, sha);
      const uint32_t x4 = (qa ^ __funnelshift_r(b_lo, b_hi, shb)) << 2;
      GZB_WALK_CHUNK(x4, qa)
      if (INC > 0) {
        a_lo = a_hi;
        b_lo = b_hi;
        pa += 1;
        pb += 1;
        a_hi = __ldg(pa + 1);
        b_hi = __ldg(pb + 1);
      } else {
        a_hi = a_lo;
        b_hi = b_lo;
        pa -= 1;
        pb -= 1;
        a_lo = __ldg(pa);
        b_lo = __ldg(pb);
      }
    }
  }
#undef GZB_WALK_CHUNK
replay : {
  // the chunk the walk ends in, pair by pair (it ends at one of them)
  int v = 0;
#define GZB_WALK_PAIR(J)                                                       \
  v = GZB_WALK_V(J, rx4, rqa);                                                 \
  score += v;                                                                  \
  best = imax(best, score);                                                    \
  if (best - score >= cutoff || best > stop_above) {                           \
    n += (J) + 1;                                                              \
    goto done;                                                                 \
  }
  GZB_WALK_PAIR(0)
  GZB_WALK_PAIR(1)
  GZB_WALK_PAIR(2)
  GZB_WALK_PAIR(3)
#undef GZB_WALK_PAIR
#undef GZB_WALK_V
done:
  *steps += n - (v == kWalkDelim ? 1 : 0);
  return best;
}
}

// One side of SeedSearcher::UngappedExtend (src/seed_searcher.h:133-158 with
// UngappedExtender::ExtendOneSideScoreOnly, src/ungapped_extender.h:34-82)
// from s0[0]/s1[0] (query/database) stepping by INC: returns the best prefix
// score, stopping at the X-drop (best - score >= cutoff, cutoff >= 1), at a
// delimiter, or once the best exceeds stop_above.  The reference's
// (best, run) pair is (best, score - best) here.  Reads four residue pairs
// per pair of aligned 32-bit words.  The first kWalkPrefetch chunks' words
// are loaded together up front (most walks end inside them, so a walk waits
// for one round of loads instead of one per chunk); a longer walk goes on
// one word per chunk.  The sequences carry delimiter padding of at least
// 4 (kWalkPrefetch + 1) bytes on each side.  *steps counts pairs examined.
template <int INC>
__device__ __forceinline__ int walk_side(const uint8_t *s0, const uint8_t *s1,
                                         const char *tbl, int cutoff, int stop_above,
                                         int *steps) {
  WalkWords<INC> A, B;
  load_walk_words(A, s0);
  load_walk_words(B, s1);
  return walk_side_words(A, B, tbl, cutoff, stop_above, steps);
}

// Whether the X-drop walk from s0[0]/s1[0] stepping by INC survives its
// first `length` residue pairs: no pair among them is a delimiter, and the
// score never falls `cutoff` (>= 1) below its running best (from 0) after
// one of them.  This is ChainFilter::Connected's back-extension
// (src/chain_filter.cpp:60-99) toward a chain end `length` pairs away,
// four pairs per chunk on the walk table (a chunk in which the walk ends
// ends it before `length`, so its exact pair does not matter).
template <int INC>
__device__ __forceinline__ bool walk_reaches(const uint8_t *s0, const uint8_t *s1,
                                             const char *tbl, int cutoff, uint32_t length) {
  const uintptr_t a0 = (uintptr_t)s0 - (INC > 0 ? 0 : 3);
  const uintptr_t a1 = (uintptr_t)s1 - (INC > 0 ? 0 : 3);
  const uint32_t *pa = (const uint32_t *)(a0 & ~(uintptr_t)3);
  const uint32_t *pb = (const uint32_t *)(a1 & ~(uintptr_t)3);
  const uint32_t sha = 8u * (uint32_t)(a0 & 3), shb = 8u * (uint32_t)(a1 & 3);
  uint32_t a_lo = __ldg(pa), a_hi = __ldg(pa + 1), b_lo = __ldg(pb), b_hi = __ldg(pb + 1);
  int score = 0, best = 0;
  uint32_t done = 0;
#define GZB_REACH_V(J, X4, QA) \
  (*(const int32_t *)(tbl + walk_offset<(INC > 0 ? (J) : 3 - (J))>(X4, QA)))
  for (;;) {
    const uint32_t qa = __funnelshift_r(a_lo, a_hi, sha);
    const uint32_t x4 = (qa ^ __funnelshift_r(b_lo, b_hi, shb)) << 2;
    if (done + 4 > length) {
      // the last pairs before the chain end, one at a time
      const uint32_t left = length - done;
#pragma unroll
      for (uint32_t j = 0; j < 3; ++j) {
        if (j >= left) break;
        const int v = j == 0 ? GZB_REACH_V(0, x4, qa)
                             : (j == 1 ? GZB_REACH_V(1, x4, qa) : GZB_REACH_V(2, x4, qa));
        score += v;
        best = imax(best, score);
        if (best - score >= cutoff) return false;
      }
      return true;
    }
    const int s0v = score + GZB_REACH_V(0, x4, qa), b0 = imax(best, s0v);
    const int s1v = s0v + GZB_REACH_V(1, x4, qa), b1 = imax(b0, s1v);
    const int s2v = s1v + GZB_REACH_V(2, x4, qa), b2 = imax(b1, s2v);
    const int s3v = s2v + GZB_REACH_V(3, x4, qa), b3 = imax(b2, s3v);
    if (imax(imax(b0 - s0v, b1 - s1v), imax(b2 - s2v, b3 - s3v)) >= cutoff) return false;
    score = s3v;
    best = b3;
    done += 4;
    if (INC > 0) {
      a_lo = a_hi;
      b_lo = b_hi;
      pa += 1;
      pb += 1;
      a_hi = __ldg(pa + 1);
      b_hi = __ldg(pb + 1);
    } else {
      a_hi = a_lo;
      b_hi = b_lo;
      pa -= 1;
      pb -= 1;
      a_lo = __ldg(pa);
      b_lo = __ldg(pb);
    }
  }
#undef GZB_REACH_V
}

// SeedSearcher::UngappedExtend on the walk table: reverse from (q-1, d-1),
// forward from (q, d) unless the reverse best already exceeds trigger; true
// when the sum exceeds trigger.
__device__ __forceinline__ bool walk_hit(const uint8_t *q, const uint8_t *d, const char *tbl,
                                         int cutoff, int trigger, int *steps) {
  int sum = walk_side<-1>(q - 1, d - 1, tbl, cutoff, trigger, steps);
  if (sum > trigger) return true;
  sum += walk_side<1>(q, d, tbl, cutoff, trigger - sum, steps);
  return sum > trigger;
}

// Reduced-alphabet mismatches over the L window centred on the seeds.
__device__ __forceinline__ int window_distance(const uint8_t *q, const uint8_t *d,
                                               int L, const uint8_t *map) {
  const int half = L / 2;
  int m = 0;
  for (int i = 0; i < L; ++i) m += map[q[i - half]] != map[d[i - half]];
  return m;
}

// ---------------------------------------------------------------------------
// Gapped extension.
struct GappedJob {
  const uint8_t *query;     // concatenated queries
  const uint8_t *db;        // database chunk
  int delim, gap_open, gap_ext, cutoff;
};

// Tile of the presearch: the gapped stage's one-thread-per-extension kernel
// (GZB_GAPPED_KERNEL_*), the flat kernel's bookkeeping threshold, whether
// the batched schedule orders extensions by the cost model (GZB_ORDER_MODEL)
// or keeps hit order (GZB_ORDER_HITS), and the seed search's walker (one
// lane per seed-search unit, GZB_SEED_WALKER_UNIT; or the unit batch's seeds
// dealt to the lanes, GZB_SEED_WALKER_DEALT), and the rows kernel's band
// columns per lane (GZB_TILE_BAND_WIDTH: 32, 64 or 128).
struct GappedTile {
  int kernel;
  int book_threshold;
  int order;
  int seed_walker;
  int band_width;
};

struct GappedOut {
  int score;
  int pos0;  // best offset along the query (negative when reversed)
  int pos1;  // best offset along the database
  uint64_t cells;
  bool overflow;
};

// Warp-cooperative first column >= c (band column numbering) whose query
// residue is the delimiter, looking at most `limit` columns ahead; returns
// c + limit when none is found.  Column c holds query residue (c-1)*inc.
__device__ __forceinline__ int find_delimiter_column(const uint8_t *q0, int inc,
                                                     int delim, int c,
                                                     int limit) {
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < limit; base += 32) {
    const int k = base + lane;
    bool is_delim = false;
    if (k < limit) is_delim = q0[(c + k - 1) * inc] == delim;
    const unsigned m = __ballot_sync(0xffffffffu, is_delim);
    if (m) return c + base + __ffs(m) - 1;
  }
  return c + limit;
}

// ---------------------------------------------------------------------------
// One extension by a group of G lanes (G = 4, 8, 16 or 32; the warp's
// 32 / G groups each run their own extension).  The same DP as
// gapped_extend_warp below, the row cut into chunks of G columns: a chunk's
// scans are G-wide shuffles within the group, and the row's running
// maximum, horizontal gap and diagonal carry over from chunk to chunk, so
// the result does not depend on G.  `band` is this group's circular buffer
// of W int2 columns; exact under the same X-drop condition.
template <int G>
struct LaneGroup {
  int lane;        // lane within the group
  int shift;       // the group's first lane within the warp
  unsigned mask;   // the group's lanes
  __device__ LaneGroup() {
    const int l = threadIdx.x & 31;
    lane = l & (G - 1);
    shift = l & ~(G - 1);
    mask = G == 32 ? 0xffffffffu : (((1u << (G & 31)) - 1u) << shift);
  }
  // the group's lanes' predicates as bits 0..G-1
  __device__ unsigned ballot(bool p) const {
    const unsigned b = __ballot_sync(mask, p) >> shift;
    return G == 32 ? b : (b & ((1u << (G & 31)) - 1u));
  }
  __device__ int up(int v, int o) const { return __shfl_up_sync(mask, v, o, G); }
  __device__ int at(int v, int src) const { return __shfl_sync(mask, v, src, G); }
  __device__ void sync() const { __syncwarp(mask); }
};

template <int G>
__device__ __forceinline__ int find_delimiter_column_group(const LaneGroup<G> &g,
                                                           const uint8_t *q0, int inc,
                                                           int delim, int c, int limit) {
  for (int base = 0; base < limit; base += G) {
    const int k = base + g.lane;
    bool is_delim = false;
    if (k < limit) is_delim = q0[(c + k - 1) * inc] == delim;
    const unsigned m = g.ballot(is_delim);
    if (m) return c + base + __ffs(m) - 1;
  }
  return c + limit;
}

template <int G, int W>
__device__ GappedOut gapped_extend_group(const GappedJob &job, const int *sm, int2 *band,
                                         uint32_t qpos, uint32_t dpos, bool reverse) {
  const LaneGroup<G> g;
  constexpr int wmask = W - 1;
  const int lane = g.lane;
  const int inc = reverse ? -1 : 1;
  const int delim = job.delim;
  const int ge = job.gap_ext;
  const int gi = job.gap_open + job.gap_ext;
  const int cutoff = job.cutoff;
  const uint8_t *q0 = job.query + qpos;
  const uint8_t *d0 = job.db + dpos;
  GappedOut out;
  out.score = 0;
  out.pos0 = -inc;
  out.pos1 = -inc;
  out.cells = 0;
  out.overflow = false;
  if (q0[0] == delim || d0[0] == delim) return out;

  // row -1: horizontal gap run from column 1 while >= -cutoff
  int k0;
  if (-gi < -cutoff) {
    k0 = 0;
  } else if (ge == 0) {
    k0 = 1 << 30;
  } else {
    long long kk = ((long long)cutoff - gi) / ge + 1;
    k0 = kk > (1 << 30) ? (1 << 30) : (int)kk;
  }
  int col = find_delimiter_column_group(g, q0, inc, delim, 1, k0 > W ? W + 1 : k0);
  if (col > W) {
    out.overflow = true;
    return out;
  }
  for (int c = 1 + lane; c < col; c += G) {
    const int s = -gi - (c - 1) * ge;
    band[c & wmask] = make_int2(s, s - gi);
  }
  if (lane == 0) band[0] = make_int2(0, -gi);
  int bs = 0, be;
  if (q0[(col - 1) * inc] != delim) {
    if (col + 1 > W) {
      out.overflow = true;
      return out;
    }
    if (lane == 0) band[col & wmask] = make_int2(kInitScore, kInitScore);
    be = col + 1;
  } else {
    be = col;
  }
  g.sync();

  int maxs = 0, mp0 = -inc, mp1 = -inc;
  uint64_t cells = 0;
  for (int r = 0;; ++r) {
    const int x = d0[r * inc];
    if (x == delim) break;
    const int *mrow = sm + x * kMatrixStride;
    const int2 st0 = band[bs & wmask];
    int diag = st0.x;
    const int nb0 = (maxs - st0.y > cutoff) ? kInitScore : st0.y;
    int F = nb0 - gi;
    g.sync();
    if (lane == 0) band[bs & wmask] = make_int2(nb0, st0.y - ge);
    int M = maxs;
    int first_kept = -1, last_kept = bs;
    for (int cs = bs + 1; cs < be; cs += G) {
      const int c = cs + lane;
      const bool active = c < be;
      int2 st = make_int2(kInitScore, kInitScore);
      int qres = 0;
      if (active) {
        st = band[c & wmask];
        qres = q0[(c - 1) * inc];
      }
      int prev = g.up(st.x, 1);
      if (lane == 0) prev = diag;
      const int Gv = imax(prev + mrow[qres], st.y);
      int P = active ? Gv - gi + (lane + 1) * ge : kNegBig;
#pragma unroll
      for (int o = 1; o < G; o <<= 1) {
        const int t = g.up(P, o);
        if (lane >= o) P = imax(P, t);
      }
      int Pex = g.up(P, 1);
      if (lane == 0) Pex = kNegBig;
      const int raw = imax(Gv, imax(F, Pex) - lane * ge);
      int R = active ? raw : kNegBig;
#pragma unroll
      for (int o = 1; o < G; o <<= 1) {
        const int t = g.up(R, o);
        if (lane >= o) R = imax(R, t);
      }
      const int Mrow = imax(M, R);
      const bool pruned = (Mrow - raw > cutoff);
      if (active) {
        const int nb = pruned ? kInitScore : raw;
        const int ng = pruned ? kInitScore : imax(raw - gi, st.y - ge);
        band[c & wmask] = make_int2(nb, ng);
      }
      const int nact = imin(G, be - cs);
      const int cm = g.at(R, G - 1);
      if (cm > M) {
        const unsigned hitm = g.ballot(active && raw == cm);
        const int l = __ffs(hitm) - 1;
        maxs = cm;
        mp0 = (cs + l - 1) * inc;
        mp1 = r * inc;
      }
      const unsigned kept = g.ballot(active && !pruned);
      if (kept) {
        if (first_kept < 0) first_kept = cs + __ffs(kept) - 1;
        last_kept = cs + 31 - __clz(kept);
      }
      const int Plast = g.at(P, nact - 1);
      F = imax(F, Plast) - nact * ge;
      M = imax(M, cm);
      diag = g.at(st.x, G - 1);
      cells += (uint64_t)nact;
    }
    g.sync();
    if (first_kept < 0) break;  // every cell pruned: array_start + 1 == array_end
    bs = first_kept - 1;
    bool edge_residue;
    if (last_kept < be - 1) {
      edge_residue = q0[(be - 1) * inc] != delim;
      be = last_kept + 1;
    } else {
      int k;
      const long long room = (long long)F - ((long long)maxs - cutoff);
      if (room < 0) {
        k = 0;
      } else if (ge == 0) {
        k = 1 << 30;
      } else {
        long long kk = room / ge + 1;
        k = kk > (1 << 30) ? (1 << 30) : (int)kk;
      }
      if (k > 0) {
        const int lim = (be + k - bs > W) ? (W - (be - bs) + 1) : k;
        k = find_delimiter_column_group(g, q0, inc, delim, be, lim) - be;
        if (be + k - bs > W) {
          out.overflow = true;
          return out;
        }
        for (int j = lane; j < k; j += G) {
          const int v = F - j * ge;
          band[(be + j) & wmask] = make_int2(v, v - gi);
        }
        be += k;
        cells += (uint64_t)k;
      }
      edge_residue = q0[(be - 1) * inc] != delim;
    }
    if (edge_residue) {
      if (be + 1 - bs > W) {
        out.overflow = true;
        return out;
      }
      if (lane == 0) band[be & wmask] = make_int2(kInitScore, kInitScore);
      ++be;
    }
    g.sync();
  }
  out.score = maxs;
  out.pos0 = mp0;
  out.pos1 = mp1;
  out.cells = cells;
  return out;
}

// One extension by one full warp.  `band` is a circular buffer of W int2
// (x = best, y = best_gap) when W > 0; the caller guarantees exactness
// conditions on the X-drop (see file comment).
template <int W>
__device__ GappedOut gapped_extend_warp(const GappedJob &job, const int *sm,
                                        int2 *band, int wmask,
                                        uint32_t qpos, uint32_t dpos,
                                        bool reverse) {
  const int lane = threadIdx.x & 31;
  const int inc = reverse ? -1 : 1;
  const int delim = job.delim;
  const int ge = job.gap_ext;
  const int gi = job.gap_open + job.gap_ext;
  const int cutoff = job.cutoff;
  const uint8_t *q0 = job.query + qpos;
  const uint8_t *d0 = job.db + dpos;
  GappedOut out;
  out.score = 0;
  out.pos0 = -inc;
  out.pos1 = -inc;
  out.cells = 0;
  out.overflow = false;
  if (q0[0] == delim || d0[0] == delim) return out;

  // Row -1: horizontal gap run from column 1 while >= -cutoff
  // (src/gapped_extender.cpp:345-364).
  int k0;
  if (-gi < -cutoff) {
    k0 = 0;
  } else if (ge == 0) {
    k0 = 1 << 30;
  } else {
    long long kk = ((long long)cutoff - gi) / ge + 1;
    k0 = kk > (1 << 30) ? (1 << 30) : (int)kk;
  }
  // stop at the delimiter
  int col = find_delimiter_column(q0, inc, delim, 1, k0 > W ? W + 1 : k0);
  if (col > W) {  // band [0, col) must fit the circular buffer
    out.overflow = true;
    return out;
  }
  const int init_cols = col - 1;  // columns 1..init_cols
  for (int c = 1 + lane; c <= init_cols; c += 32) {
    const int s = -gi - (c - 1) * ge;
    band[c & wmask] = make_int2(s, s - gi);
  }
  if (lane == 0) band[0] = make_int2(0, -gi);
  int bs = 0, be;
  if (q0[(col - 1) * inc] != delim) {
    if (col + 1 > W) {
      out.overflow = true;
      return out;
    }
    if (lane == 0) band[col & wmask] = make_int2(kInitScore, kInitScore);
    be = col + 1;
  } else {
    be = col;
  }
  __syncwarp();

  int maxs = 0, mp0 = -inc, mp1 = -inc;
  uint64_t cells = 0;
  for (int r = 0;; ++r) {
    const int x = d0[r * inc];
    if (x == delim) break;
    const int *mrow = sm + x * kMatrixStride;
    // column bs: vertical gap only (src/gapped_extender.cpp:397-408)
    const int2 st0 = band[bs & wmask];
    int diag = st0.x;
    const int nb0 = (maxs - st0.y > cutoff) ? kInitScore : st0.y;
    int F = nb0 - gi;
    __syncwarp();
    if (lane == 0) band[bs & wmask] = make_int2(nb0, st0.y - ge);
    int M = maxs;
    int first_kept = -1, last_kept = bs;
    for (int cs = bs + 1; cs < be; cs += 32) {
      const int c = cs + lane;
      const bool active = c < be;
      int2 st = make_int2(kInitScore, kInitScore);
      int qres = 0;
      if (active) {
        st = band[c & wmask];
        qres = q0[(c - 1) * inc];
      }
      int prev = __shfl_up_sync(0xffffffffu, st.x, 1);
      if (lane == 0) prev = diag;
      const int G = imax(prev + mrow[qres], st.y);
      // F: exclusive max-plus scan of B(j) = G(j) - gi + (j+1)*ge
      int P = active ? G - gi + (lane + 1) * ge : kNegBig;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, P, o);
        if (lane >= o) P = imax(P, t);
      }
      int Pex = __shfl_up_sync(0xffffffffu, P, 1);
      if (lane == 0) Pex = kNegBig;
      const int Fl = imax(F, Pex) - lane * ge;
      const int raw = imax(G, Fl);
      // running maximum: inclusive prefix max of raw
      int R = active ? raw : kNegBig;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, R, o);
        if (lane >= o) R = imax(R, t);
      }
      const int Mrow = imax(M, R);
      const bool pruned = (Mrow - raw > cutoff);
      if (active) {
        const int nb = pruned ? kInitScore : raw;
        const int ng = pruned ? kInitScore : imax(raw - gi, st.y - ge);
        band[c & wmask] = make_int2(nb, ng);
      }
      const int nact = imin(32, be - cs);
      // new maximum: first column reaching the chunk maximum
      const int cm = __shfl_sync(0xffffffffu, R, 31);
      if (cm > M) {
        const unsigned hitm = __ballot_sync(0xffffffffu, active && raw == cm);
        const int l = __ffs(hitm) - 1;
        maxs = cm;
        mp0 = (cs + l - 1) * inc;
        mp1 = r * inc;
      }
      const unsigned kept = __ballot_sync(0xffffffffu, active && !pruned);
      if (kept) {
        if (first_kept < 0) first_kept = cs + __ffs(kept) - 1;
        last_kept = cs + 31 - __clz(kept);
      }
      // carries into the next chunk / the band-extension step
      const int Plast = __shfl_sync(0xffffffffu, P, nact - 1);
      F = imax(F, Plast) - nact * ge;
      M = imax(M, cm);
      diag = __shfl_sync(0xffffffffu, st.x, 31);
      cells += (uint64_t)nact;
    }
    __syncwarp();
    if (first_kept < 0) break;  // every cell pruned: array_start + 1 == array_end
    bs = first_kept - 1;
    bool edge_residue;
    if (last_kept < be - 1) {
      // shrink; the reference tests the residue of the old right edge
      edge_residue = q0[(be - 1) * inc] != delim;
      be = last_kept + 1;
    } else {
      // grow along the horizontal gap while F >= max - cutoff
      int k;
      const long long room = (long long)F - ((long long)maxs - cutoff);
      if (room < 0) {
        k = 0;
      } else if (ge == 0) {
        k = 1 << 30;
      } else {
        long long kk = room / ge + 1;
        k = kk > (1 << 30) ? (1 << 30) : (int)kk;
      }
      if (k > 0) {
        const int lim = (be + k - bs > W) ? (W - (be - bs) + 1) : k;
        k = find_delimiter_column(q0, inc, delim, be, lim) - be;
        if (be + k - bs > W) {
          out.overflow = true;
          return out;
        }
        for (int j = lane; j < k; j += 32) {
          const int v = F - j * ge;
          band[(be + j) & wmask] = make_int2(v, v - gi);
        }
        be += k;
        cells += (uint64_t)k;
      }
      edge_residue = q0[(be - 1) * inc] != delim;
    }
    if (edge_residue) {
      if (be + 1 - bs > W) {
        out.overflow = true;
        return out;
      }
      if (lane == 0) band[be & wmask] = make_int2(kInitScore, kInitScore);
      ++be;
    }
    __syncwarp();
  }
  out.score = maxs;
  out.pos0 = mp0;
  out.pos1 = mp1;
  out.cells = cells;
  return out;
}

}  // namespace gzb

namespace gzb {

// Serial restatement of the same extension for one thread, with the band in
// a circular global buffer of wmask+1 columns.  Exact for every X-drop; used
// for extensions whose band outgrows the warp kernel's shared buffer and for
// X-drops in [1024, 2^30).  Sets *too_long when the band would exceed the
// buffer (the caller reports GZB_ERR_OVERFLOW).
__device__ inline GappedOut gapped_extend_serial(const GappedJob &job,
                                                 const int *sm, int2 *band,
                                                 int wmask, uint32_t qpos,
                                                 uint32_t dpos, bool reverse,
                                                 bool *too_long) {
  const int inc = reverse ? -1 : 1;
  const int delim = job.delim;
  const int ge = job.gap_ext;
  const int gi = job.gap_open + job.gap_ext;
  const int cutoff = job.cutoff;
  const int W = wmask + 1;
  const uint8_t *q0 = job.query + qpos;
  const uint8_t *d0 = job.db + dpos;
  GappedOut out;
  out.score = 0;
  out.pos0 = -inc;
  out.pos1 = -inc;
  out.cells = 0;
  out.overflow = false;
  *too_long = false;
  if (q0[0] == delim || d0[0] == delim) return out;
  int score = -gi;
  int col = 1;
  int p0 = 0;
  band[0] = make_int2(0, -gi);
  for (; q0[p0] != delim; ++col, p0 += inc) {
    if (score < -cutoff) break;
    if (col >= W) {
      *too_long = true;
      return out;
    }
    band[col & wmask] = make_int2(score, score - gi);
    score -= ge;
  }
  int bs = 0, be;
  if (q0[p0] != delim) {
    if (col >= W) {
      *too_long = true;
      return out;
    }
    band[col & wmask] = make_int2(kInitScore, kInitScore);
    be = col + 1;
  } else {
    be = col;
  }
  int maxs = 0, mp0 = -inc, mp1 = -inc;
  uint64_t cells = 0;
  for (int p1 = 0; d0[p1] != delim; p1 += inc) {
    const int *mrow = sm + d0[p1] * kMatrixStride;
    p0 = bs * inc;
    int2 *c0 = &band[bs & wmask];
    int diag = c0->x;
    c0->x = (maxs - c0->y > cutoff) ? kInitScore : c0->y;
    int row_gap = c0->x - gi;
    c0->y -= ge;
    int last = bs;
    const int bs_row = bs;
    for (int c = bs_row + 1; c < be; ++c, p0 += inc) {
      int2 *cell = &band[c & wmask];
      int s = diag + mrow[q0[p0]];
      diag = cell->x;
      const int vgap = cell->y;
      ++cells;
      if (s < vgap) s = vgap;
      if (s < row_gap) s = row_gap;
      if (maxs - s > cutoff) {
        if (bs + 1 == c) ++bs;
        cell->x = kInitScore;
        cell->y = kInitScore;
        row_gap = kInitScore;
      } else {
        last = c;
        if (s > maxs) {
          maxs = s;
          mp0 = p0;
          mp1 = p1;
        }
        cell->y = imax(s - gi, vgap - ge);
        row_gap = imax(s - gi, row_gap - ge);
        cell->x = s;
      }
    }
    if (bs + 1 == be) break;
    if (last < be - 1) {
      be = last + 1;
    } else {
      while (row_gap >= maxs - cutoff && q0[p0] != delim) {
        if (be - bs >= W) {
          *too_long = true;
          return out;
        }
        band[be & wmask] = make_int2(row_gap, row_gap - gi);
        row_gap -= ge;
        ++be;
        p0 += inc;
        ++cells;
      }
    }
    if (q0[p0] != delim) {
      if (be - bs >= W) {
        *too_long = true;
        return out;
      }
      band[be & wmask] = make_int2(kInitScore, kInitScore);
      ++be;
    }
  }
  out.score = maxs;
  out.pos0 = mp0;
  out.pos1 = mp1;
  out.cells = cells;
  return out;
}

// True when the warp kernel's no-reset scan is exact for this X-drop.
__host__ __device__ inline bool warp_path_exact(int cutoff) {
  return cutoff < 1024 || cutoff >= (1 << 30);
}

}  // namespace gzb

namespace gzb {

// ---------------------------------------------------------------------------
// Gapped extension, one thread per extension (the common, narrow-band case).
// The exact serial recurrence of GappedExtender::ExtendOneSideScoreOnly with
// the band in shared memory: W columns per thread (a power of two; kLaneW
// unless the rows kernel's band-width tile says otherwise), each a packed
// int16 pair (best, best_gap), plus the query residue of each band column
// (one byte: the residue's byte offset in a score-matrix row), laid out
// [column][thread] so that a warp touching one column
// per thread is bank-conflict free.  A band wider than W, or a value
// outside int16, makes the extension overflow; the caller reruns it on the
// warp kernel.
constexpr int kLaneW = 64;

// The residue bytes of a band column are laid out so that lane l of every
// warp uses bank l: byte 4l + w of the column's 128 bytes belongs to lane l
// of warp w (blocks of four warps), so the lanes of a warp never conflict,
// whatever columns they are at (with the plain [column][thread] byte layout
// four lanes share each bank).
template <int W = kLaneW>
struct LaneBand {
  static_assert(W >= 8 && (W & (W - 1)) == 0, "the band width is a power of two");
  static constexpr int kW = W;
  uint32_t *cell;  // [W][stride]
  uint8_t *res;    // [W][stride], lane-major within a column
  int stride;      // threads of the block (128)
  int t;           // this thread's column in the cell layout
  int tr;          // this thread's byte in the residue layout
  __device__ __forceinline__ LaneBand(uint32_t *cell_, uint8_t *res_, int stride_, int t_)
      : cell(cell_), res(res_), stride(stride_), t(t_), tr(((t_ & 31) << 2) | (t_ >> 5)) {}
  __device__ __forceinline__ int base(int c) const { return (c & (W - 1)) * stride; }
  __device__ __forceinline__ int slot(int c) const { return base(c) + t; }
  __device__ __forceinline__ uint32_t &at(int c) { return cell[slot(c)]; }
  // a column's query residue r is kept as its byte offset in a matrix row (4r)
  __device__ __forceinline__ void set_residue(int c, int r) {
    res[base(c) + tr] = (uint8_t)(r << 2);
  }
};

__device__ __forceinline__ bool fits16(int v) { return v >= -32768 && v <= 32767; }
__device__ __forceinline__ uint32_t pack16(int best, int gap) {
  return ((uint32_t)(uint16_t)(int16_t)best) | ((uint32_t)(uint16_t)(int16_t)gap << 16);
}
__device__ __forceinline__ int lo16(uint32_t w) { return (int)(int16_t)(uint16_t)(w & 0xffff); }
__device__ __forceinline__ int hi16(uint32_t w) { return (int)(int16_t)(uint16_t)(w >> 16); }

// State of one extension on the lane kernels, kept in registers between
// rows: band [bs, be) of absolute columns, the running maximum and its
// position, the database offset of the next row and the cell count.
struct LaneExt {
  const uint8_t *q0, *d0;
  int inc;
  int bs, be;
  int maxs, mp0, mp1;
  int p1;
  int xr;  // database residue of row p1, loaded one row ahead
  uint32_t cells;
  bool ovf;
};

enum : int { kLaneRunning = 0, kLaneDone = 1, kLaneOverflow = 2 };

// Row -1 of GappedExtender::ExtendOneSideScoreOnly
// (src/gapped_extender.cpp:345-364): the gap-open row along the query until
// it drops below -cutoff, plus the sentinel column.
template <int W>
__device__ __forceinline__ int lane_init(const GappedJob &job, LaneBand<W> &band, LaneExt &x,
                                         const uint8_t *q0, const uint8_t *d0, bool reverse) {
  const int inc = reverse ? -1 : 1;
  const int delim = job.delim;
  const int ge = job.gap_ext;
  const int gi = job.gap_open + job.gap_ext;
  x.q0 = q0;
  x.d0 = d0;
  x.inc = inc;
  x.maxs = 0;
  x.mp0 = -inc;
  x.mp1 = -inc;
  x.p1 = 0;
  x.cells = 0;
  x.ovf = false;
  x.xr = d0[0];
  if (q0[0] == delim || x.xr == delim) return kLaneDone;
  // every value a row keeps lies in [maxs - cutoff - gi, maxs] with maxs >= 0,
  // so checking maxs once per row is enough when cutoff + gi fits; the
  // values written here lie in [-cutoff - gi, 0]
  x.ovf = job.cutoff + gi > 32767;
  band.at(0) = pack16(0, -gi);
  int score = -gi;
  int col = 1;
  int r = 0;
  // query residues q0[0], q0[inc], ... four per aligned word pair
  const uintptr_t a0 = (uintptr_t)q0 - (inc > 0 ? 0 : 3);
  const uint32_t *p = (const uint32_t *)(a0 & ~(uintptr_t)3);
  const uint32_t sh = 8u * (uint32_t)(a0 & 3);
  uint32_t lo = __ldg(p), hi = __ldg(p + 1);
  for (;;) {
    uint32_t w = __funnelshift_r(lo, hi, sh);
    if (inc < 0) w = __byte_perm(w, 0, 0x0123);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      r = (int)((w >> (8 * j)) & 0xffu);
      if (r == delim || score < -job.cutoff) goto init_done;
      if (col >= W) return kLaneOverflow;
      band.at(col) = pack16(score, score - gi);
      band.set_residue(col, r);
      score -= ge;
      ++col;
    }
    if (inc > 0) {
      lo = hi;
      ++p;
      hi = __ldg(p + 1);
    } else {
      hi = lo;
      --p;
      lo = __ldg(p);
    }
  }
init_done:
  x.bs = 0;
  if (r != delim) {
    if (col >= W) return kLaneOverflow;
    band.at(col) = pack16(kInitScore, kInitScore);
    band.set_residue(col, r);
    x.be = col + 1;
  } else {
    x.be = col;
  }
  return kLaneRunning;
}

// One database row of the recurrence (src/gapped_extender.cpp:366-470):
// the cells of the band, the X-drop trimming of its left edge, and the
// right edge moving or growing along the gap row.
template <int W>
__device__ __forceinline__ int lane_row(const GappedJob &job, const int *sm, LaneBand<W> &band,
                                        LaneExt &x) {
  const int inc = x.inc;
  const int delim = job.delim;
  const int ge = job.gap_ext;
  const int gi = job.gap_open + job.gap_ext;
  const int cutoff = job.cutoff;
  const uint8_t *q0 = x.q0;
  const int p1 = x.p1;
  const int xr = x.xr;
  if (xr == delim) return kLaneDone;
  x.xr = x.d0[p1 + inc];  // the next row's residue (the chunk is padded)
  const int *mrow = sm + xr * kMatrixStride;
  int bs = x.bs, be = x.be, maxs = x.maxs;
  bool ovf = x.ovf;
  uint32_t &c0 = band.at(bs);
  const uint32_t w0 = c0;
  int diag = lo16(w0);
  const int g0 = hi16(w0);
  const int nb0 = (maxs - g0 > cutoff) ? kInitScore : g0;
  int row_gap = nb0 - gi;
  ovf |= !fits16(g0 - ge);
  c0 = pack16(nb0, g0 - ge);
  int last = bs;
  const int bs_row = bs;
  const int maxs_in = maxs;
  int maxc = bs_row;
  bool lead = true;  // every cell of the row so far pruned
  for (int c = bs_row + 1; c < be; ++c) {
    const int b = band.base(c);
    const int k = b + band.t;
    const uint32_t w = band.cell[k];
    const int old_best = lo16(w), vgap = hi16(w);
    int s = diag + *(const int *)((const char *)mrow + band.res[b + band.tr]);
    diag = old_best;
    s = imax(s, imax(vgap, row_gap));
    // branch-free: a pruned cell (X-drop) stores the initial score and resets
    // the row gap; the left edge moves past a leading run of pruned cells
    const bool drop = maxs - s > cutoff;
    lead = lead && drop;
    bs = lead ? c : bs;
    last = drop ? last : c;
    maxc = s > maxs ? c : maxc;  // a pruned cell is below maxs
    maxs = imax(maxs, s);
    const int sg = s - gi;
    const int ng = imax(sg, vgap - ge);
    row_gap = drop ? kInitScore : imax(sg, row_gap - ge);
    band.cell[k] = drop ? pack16(kInitScore, kInitScore) : pack16(s, ng);
  }
  const uint32_t cells = (uint32_t)(be - bs_row - 1);
  if (maxs > maxs_in) {
    x.mp0 = (maxc - 1) * inc;
    x.mp1 = p1;
  }
  ovf |= maxs > 32767;
  x.cells += cells;
  x.maxs = maxs;
  x.ovf = ovf;
  x.bs = bs;
  if (bs + 1 == be) return kLaneDone;
  int edge;  // residue the reference tests after the row (:461)
  if (last < be - 1) {
    edge = q0[(be - 1) * inc];  // old right edge
    be = last + 1;
  } else {
    edge = q0[(be - 1) * inc];
    while (row_gap >= maxs - cutoff && edge != delim) {
      if (be - bs >= W) return kLaneOverflow;
      x.ovf |= !fits16(row_gap) || !fits16(row_gap - gi);
      band.at(be) = pack16(row_gap, row_gap - gi);
      band.set_residue(be, edge);
      row_gap -= ge;
      ++be;
      ++x.cells;
      edge = q0[(be - 1) * inc];
    }
  }
  if (edge != delim) {
    if (be - bs >= W) return kLaneOverflow;
    band.at(be) = pack16(kInitScore, kInitScore);
    // the sentinel column's own residue (differs from `edge` when the band shrank)
    band.set_residue(be, q0[(be - 1) * inc]);
    ++be;
  }
  x.be = be;
  x.p1 = p1 + inc;
  return kLaneRunning;
}

template <int W>
__device__ inline GappedOut gapped_extend_lane(const GappedJob &job, const int *sm,
                                               LaneBand<W> band, uint32_t qpos, uint32_t dpos,
                                               bool reverse) {
  LaneExt x;
  int st = lane_init(job, band, x, job.query + qpos, job.db + dpos, reverse);
  while (st == kLaneRunning) st = lane_row(job, sm, band, x);
  GappedOut out;
  out.overflow = st == kLaneOverflow || x.ovf;
  out.score = x.maxs;
  out.pos0 = x.mp0;
  out.pos1 = x.mp1;
  out.cells = x.cells;
  return out;
}

}  // namespace gzb

namespace gzb {

// ---------------------------------------------------------------------------
// Gapped extension, one thread per extension, flattened.  Same recurrence as
// gapped_extend_lane, but the row loop, the cell loop and the loop over
// extensions are one loop that advances every lane by one DP cell per
// iteration: a lane that reaches the end of its row, or of its extension,
// does that bookkeeping and carries on with its next cell, so the lanes of a
// warp never wait for the slowest one.  Band cells are int2 {best,
// best_gap << 5 | query residue} in a kFlatW-column circular buffer per
// thread ([column][thread] layout).  Extensions whose band outgrows it, or
// that run past 2^24 rows (the packed gap field's bound), are handed on.
constexpr int kFlatW = 48;
constexpr int kFlatBlock = 128;

struct FlatOut {
  uint32_t *qpos, *dpos;
  int32_t *scores;
  uint32_t *spill, *spill_count;
  uint32_t *cells_out;  // optional, per extension (UINT32_MAX when handed on)
};

__device__ __forceinline__ int flat_next(int s) { return s + 1 == kFlatW ? 0 : s + 1; }
__device__ __forceinline__ int pack_gap(int gap, int res) {
  return (int)(((uint32_t)gap << 5) | (uint32_t)res);
}

// Work source: queue (device counter over `n` items, optionally through
// `order`).  Returns false when exhausted.
__device__ __forceinline__ bool flat_fetch(unsigned long long *queue, uint64_t n,
                                           const uint32_t *order, uint32_t *e) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(queue, (unsigned long long)g.size());
  base = g.shfl(base, 0);
  const unsigned long long i = base + g.thread_rank();
  if (i >= n) return false;
  *e = order ? order[i] : (uint32_t)i;
  return true;
}

__device__ __forceinline__ unsigned long long gapped_flat(const GappedJob &job, const int *sm,
                                                          int2 *band, int S, uint64_t n,
                                                          const uint32_t *order,
                                                          unsigned long long *queue,
                                                          int reverse_default,
                                                          const uint8_t *dir, FlatOut out,
                                                          int book_threshold) {
  const int delim = job.delim;
  const int ge = job.gap_ext;
  const int gi = job.gap_open + job.gap_ext;
  const int cutoff = job.cutoff;
  unsigned long long cells_total = 0;
  // per-lane state
  uint32_t e = 0;
  int inc = 1;
  const uint8_t *q0 = nullptr, *d0 = nullptr;
  int bs = 0, be = 0, bss = 0, bes = 0;   // band [bs, be) and the slots of bs / be
  int c = 0, cs = 0, pos0 = 0;            // current column, its slot, its query offset
  int last = 0, ls = 0;                   // last kept column and its slot
  int diag = 0, row_gap = 0;
  int maxs = 0, mp0 = 0, mp1 = 0;
  int r = 0, p1 = 0, next_x = 0;
  const int *mrow = sm;
  uint32_t cells = 0;
  bool have = false, done = false;
  for (;;) {
    // Every iteration starts with the whole warp converged.  Lanes that
    // reached a row or extension boundary wait until at least
    // `book_threshold` of them do (or no lane can take a cell step) and then
    // do their bookkeeping together, so the long bookkeeping path runs with
    // many lanes at once instead of with one lane per iteration.
    __syncwarp();
    const bool cell_ready = have && !done && c < be;
    const bool book_ready = !done && !cell_ready;
    const unsigned cm = __ballot_sync(0xffffffffu, cell_ready);
    const unsigned bm = __ballot_sync(0xffffffffu, book_ready);
    if ((cm | bm) == 0) break;
    const bool book_turn = cm == 0 || __popc(bm) >= book_threshold;
    if (!book_turn) {
      if (!cell_ready) continue;
      // ---- one DP cell (src/gapped_extender.cpp:410-443)
      int2 &cell = band[cs * S];
      const int2 w = cell;
      const int res = w.y & 31;
      const int vgap = w.y >> 5;
      int s = diag + mrow[res];
      diag = w.x;
      s = imax(s, imax(vgap, row_gap));
      ++cells;
      if (maxs - s > cutoff) {
        if (bs + 1 == c) {
          bs = c;
          bss = cs;
        }
        cell = make_int2(kInitScore, pack_gap(kInitScore, res));
        row_gap = kInitScore;
      } else {
        last = c;
        ls = cs;
        if (s > maxs) {
          maxs = s;
          mp0 = pos0;
          mp1 = p1;
        }
        const int ng = imax(s - gi, vgap - ge);
        row_gap = imax(s - gi, row_gap - ge);
        cell = make_int2(s, pack_gap(ng, res));
      }
      ++c;
      pos0 += inc;
      cs = flat_next(cs);
      continue;
    }
    if (!book_ready) continue;
    // ---- bookkeeping: row end, next row, next extension
    bool finish = false, overflow = false;
    if (have) {
      // row end (src/gapped_extender.cpp:445-465)
      if (bs + 1 == be) {
        finish = true;
      } else {
        int edge;
        const bool shrunk = last < be - 1;
        if (shrunk) {
          edge = q0[(be - 1) * inc];  // the old right edge is tested
          be = last + 1;
          bes = flat_next(ls);
        } else {
          edge = q0[(be - 1) * inc];
          while (row_gap >= maxs - cutoff && edge != delim) {
            if (be - bs >= kFlatW) {
              overflow = true;
              break;
            }
            band[bes * S] = make_int2(row_gap, pack_gap(row_gap - gi, edge));
            row_gap -= ge;
            ++be;
            bes = flat_next(bes);
            ++cells;
            edge = q0[(be - 1) * inc];
          }
        }
        if (!overflow && edge != delim) {
          if (be - bs >= kFlatW) {
            overflow = true;
          } else {
            // the sentinel column keeps its own residue
            const int res = shrunk ? (band[bes * S].y & 31) : edge;
            band[bes * S] = make_int2(kInitScore, pack_gap(kInitScore, res));
            ++be;
            bes = flat_next(bes);
          }
        }
        ++r;
        p1 += inc;
      }
    }
    for (;;) {
      if (have && !finish && !overflow) {
        // row start (src/gapped_extender.cpp:382-408)
        const int x = next_x;
        if (x == delim) {
          finish = true;
        } else if (r >= (1 << 24)) {
          overflow = true;
        } else {
          next_x = d0[p1 + inc];
          mrow = sm + x * kMatrixStride;
          int2 &c0 = band[bss * S];
          const int2 w0 = c0;
          const int g0 = w0.y >> 5;
          diag = w0.x;
          const int nb0 = (maxs - g0 > cutoff) ? kInitScore : g0;
          row_gap = nb0 - gi;
          c0 = make_int2(nb0, pack_gap(g0 - ge, w0.y & 31));
          last = bs;
          ls = bss;
          c = bs + 1;
          cs = flat_next(bss);
          pos0 = bs * inc;
          break;  // back to cell steps
        }
      }
      if (have) {
        if (overflow) {
          out.spill[atomicAdd(out.spill_count, 1u)] = e;
          if (out.cells_out) out.cells_out[e] = 0xFFFFFFFFu;
        } else {
          const uint32_t q = out.qpos[e], d = out.dpos[e];
          out.qpos[e] = q + (uint32_t)mp0;
          out.dpos[e] = d + (uint32_t)mp1;
          out.scores[e] = maxs;
          if (out.cells_out) out.cells_out[e] = cells;
          cells_total += cells;
        }
        have = false;
      }
      // next extension
      if (!flat_fetch(queue, n, order, &e)) {
        done = true;
        break;
      }
      have = true;
      finish = false;
      overflow = false;
      const bool rev = dir ? dir[e] != 0 : reverse_default != 0;
      inc = rev ? -1 : 1;
      q0 = job.query + out.qpos[e];
      d0 = job.db + out.dpos[e];
      maxs = 0;
      mp0 = -inc;
      mp1 = -inc;
      cells = 0;
      r = 0;
      p1 = 0;
      if (q0[0] == delim || d0[0] == delim) {
        finish = true;
        continue;
      }
      // row -1 (src/gapped_extender.cpp:345-364)
      band[0] = make_int2(0, pack_gap(-gi, 0));
      int score = -gi, col = 1, res = q0[0];
      for (;;) {
        if (res == delim || score < -cutoff) break;
        if (col >= kFlatW) {
          overflow = true;
          break;
        }
        band[col * S] = make_int2(score, pack_gap(score - gi, res));
        score -= ge;
        ++col;
        res = q0[(col - 1) * inc];
      }
      if (overflow) continue;
      if (res != delim) {
        if (col >= kFlatW) {
          overflow = true;
          continue;
        }
        band[col * S] = make_int2(kInitScore, pack_gap(kInitScore, res));
        be = col + 1;
      } else {
        be = col;
      }
      bs = 0;
      bss = 0;
      bes = be == kFlatW ? 0 : be;
      next_x = d0[0];
    }
  }
  return cells_total;
}

}  // namespace gzb
