// gzb_traceback.cu -- alignment statistics of the merged results (the build
// results step): both sides of every result of the resident chunk are
// extended again with their edit path, and the path yields the figures
// AlignerCommon::BuildResult reports (alignment length, mismatches, gap
// openings and extensions).
//
// One warp per side runs the DP once, storing one op byte per cell row by
// row in the warp's own scratch (so no pass sizes the storage first),
// walks the optimal path back from the best cell (PickOptimalPath) and
// counts what BuildResult counts over it; a last kernel joins the two sides
// of each result in the reference's order.
//
// The warp evaluates 32 consecutive columns of a row at once, with the
// presearch's warp DP (gapped_extend_warp in gzb_kernels.cuh: band edges and
// stored values exact for X-drops below 1024).  A kept cell's edit op also
// needs the reference's horizontal-gap value *with* its reset to
// kInitScore at pruned cells (src/gapped_extender.cpp:428-446); once a
// chunk's pruned flags are known that value is a segmented max-plus scan
// whose segments start after the pruned cells.  Sides whose band outgrows
// the warp's circular buffer, whose storage outgrows the warp's scratch, or
// whose X-drop is 1024 or more are flagged and run by one thread each: a
// pass to size their storage, then the DP with the band in global memory
// (the serial form of the same DP), the walk and the counts.
#include <cuda_runtime.h>

#include <cstdint>

#include "ghostz_b200.h"
#include "gzb_common.h"
#include "gzb_kernels.cuh"
#include "gzb_traceback.cuh"

namespace gzb {

namespace {

// edit ops of the DP (src/gapped_extender.h:46-52)
constexpr int kTbSub = 0, kTbGap0 = 1, kTbGap1 = 2, kTbExt0 = 4, kTbExt1 = 8;
// ops of the path, EditBlocks numbering (src/edit_blocks.h:14-18)
constexpr uint8_t kPathGap0 = 0, kPathSub = 1, kPathGap1 = 2;

struct TbSide {
  const uint8_t *seq0, *seq1;
  int inc;
  uint32_t len0;  // residues of seq0 before its delimiter
  bool active;
};

__device__ TbSide side_of(const TbArgs &a, uint64_t side) {
  TbSide t;
  const uint64_t slot = side >> 1;
  const bool fwd = (side & 1) != 0;
  const uint32_t qi = (uint32_t)(slot / (uint64_t)a.max_results);
  const uint32_t k = (uint32_t)(slot % (uint64_t)a.max_results);
  t.active = false;
  t.seq0 = t.seq1 = nullptr;
  t.inc = fwd ? 1 : -1;
  t.len0 = 0;
  if (qi >= a.nq || k >= a.counts[qi]) return t;
  const gzb_result r = a.results[slot];
  if (r.chunk_id != a.chunk_id || r.hit_q == 0) return t;
  const uint8_t *qs = a.query + a.q_offsets[qi];
  t.active = true;
  if (fwd) {
    t.seq0 = qs + r.hit_q;
    t.seq1 = a.db + r.hit_d;
    t.len0 = a.q_lengths[qi] - 1 - r.hit_q;
  } else {
    t.seq0 = qs + r.hit_q - 1;
    t.seq1 = a.db + r.hit_d - 1;
    t.len0 = r.hit_q - 1;
  }
  return t;
}

// GappedExtender::ExtendOneSide (src/gapped_extender.cpp:70-304) with the
// band in global memory (cell[col] = {best, best_gap}, len0 + 2 columns).
// With `ops` null it only counts: *ops_bytes = the row storage the reference
// keeps (final band end - band start, per row), *rows = rows stored.
// Otherwise row r's op of column c goes to ops[row_meta[2r] + c -
// row_meta[2r + 1]] (ops must be zeroed: a cell the DP prunes keeps 0).
__device__ void tb_extend(const TbArgs &a, const int *sm, const TbSide &t, int2 *cell,
                          uint8_t *ops, uint32_t *row_meta, uint64_t *ops_bytes,
                          uint32_t *rows, int *best_score, int *best_p0, int *best_p1) {
  const int inc = t.inc;
  const int delim = a.delim;
  const int ge = a.gap_ext;
  const int gi = a.gap_open + a.gap_ext;
  const int cutoff = a.cutoff;
  const uint8_t *seq0 = t.seq0, *seq1 = t.seq1;
  *best_score = 0;
  *best_p0 = -inc;
  *best_p1 = -inc;
  *ops_bytes = 0;
  *rows = 0;
  if (seq0[0] == delim || seq1[0] == delim) return;
  int score = -gi, col = 1, pos0 = 0;
  cell[0] = make_int2(0, -gi);
  for (; seq0[pos0] != delim; ++col, pos0 += inc) {
    if (score < -cutoff) break;
    cell[col] = make_int2(score, score - gi);
    score -= ge;
  }
  int bs = 0, be;
  if (seq0[pos0] != delim) {
    cell[col] = make_int2(kInitScore, kInitScore);
    be = col + 1;
  } else {
    be = col;
  }
  int max_score = 0, max_p0 = -inc, max_p1 = -inc;
  uint64_t used = 0;
  uint32_t r = 0;
  for (int pos1 = 0; seq1[pos1] != delim; pos1 += inc, ++r) {
    const int *mrow = sm + seq1[pos1] * kMatrixStride;
    const int row_start = bs;
    uint8_t *row_ops = nullptr;
    if (ops) {
      row_meta[2 * r] = (uint32_t)used;
      row_meta[2 * r + 1] = (uint32_t)row_start;
      row_ops = ops + used - row_start;
    }
    pos0 = bs * inc;
    const int2 c0 = cell[bs];
    int diag = c0.x;
    const int nb = (max_score - c0.y > cutoff) ? kInitScore : c0.y;
    int row_gap = nb - gi;
    cell[bs] = make_int2(nb, c0.y - ge);
    if (ops) row_ops[bs] = kTbGap0 + kTbExt0;
    int last = bs;
    for (col = bs + 1; col < be; ++col, pos0 += inc) {
      const int2 w = cell[col];
      int s = diag + mrow[seq0[pos0]];
      const int vgap = w.y;
      diag = w.x;
      int op = kTbSub;
      if (s < vgap) {
        op = kTbGap0;
        s = vgap;
      }
      if (s < row_gap) {
        op = kTbGap1;
        s = row_gap;
      }
      if (max_score - s > cutoff) {
        if (bs + 1 == col) ++bs;
        cell[col] = make_int2(kInitScore, kInitScore);
        row_gap = kInitScore;
      } else {
        last = col;
        if (s > max_score) {
          max_score = s;
          max_p0 = pos0;
          max_p1 = pos1;
        }
        int ng;
        if (vgap - ge < s - gi) {
          ng = s - gi;
        } else {
          ng = vgap - ge;
          op += kTbExt0;
        }
        if (row_gap - ge < s - gi) {
          row_gap = s - gi;
        } else {
          row_gap -= ge;
          op += kTbExt1;
        }
        if (ops) row_ops[col] = (uint8_t)op;
        cell[col] = make_int2(s, ng);
      }
    }
    if (bs + 1 == be) {
      ++r;
      break;
    }
    if (last < be - 1) {
      be = last + 1;
    } else {
      while (row_gap >= max_score - cutoff && seq0[pos0] != delim) {
        cell[be] = make_int2(row_gap, row_gap - gi);
        if (ops) row_ops[be] = kTbGap0 + kTbExt0;
        row_gap -= ge;
        ++be;
        pos0 += inc;
      }
    }
    if (seq0[pos0] != delim) {
      cell[be] = make_int2(kInitScore, kInitScore);
      ++be;
    }
    used += (uint64_t)(be - row_start);  // the reference's row accounting (:464-466)
  }
  // the row the DP stopped in keeps its ops too
  *ops_bytes = used + (uint64_t)(t.len0 + 2);
  *rows = r;
  *best_score = max_score;
  *best_p0 = max_p0;
  *best_p1 = max_p1;
}

constexpr int kTbWarpColumns = 256;  // circular band of one warp (int2 columns)
constexpr int kTbWarpsPerBlock = 8;
static_assert(kTbWarpBlock == kTbWarpsPerBlock * 32, "launch block of the warp kernels");

// tb_extend by one warp (lanes must all call it with the same side); with
// STORE it also writes the ops and row table as tb_extend does, into
// storage of ops_cap bytes and rows_cap rows that need not be zeroed: every
// byte of a row's range is written (0 for a pruned cell and the sentinel,
// as a fresh GappedExtender holds), and the bytes past the last row up to
// *ops_bytes are zeroed at the end.  Returns false when the band outgrows
// kTbWarpColumns or the side outgrows the storage (outputs then
// meaningless).
template <bool STORE>
__device__ bool tb_extend_warp(const TbArgs &a, const int *sm, const TbSide &t, int2 *band,
                               uint8_t *ops, uint32_t *row_meta, uint64_t ops_cap,
                               uint32_t rows_cap, uint64_t *ops_bytes, uint32_t *rows,
                               int *best_score, int *best_p0, int *best_p1) {
  constexpr int W = kTbWarpColumns;
  constexpr int wmask = W - 1;
  constexpr unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int inc = t.inc;
  const int delim = a.delim;
  const int ge = a.gap_ext;
  const int gi = a.gap_open + a.gap_ext;
  const int cutoff = a.cutoff;
  const uint8_t *q0 = t.seq0, *d0 = t.seq1;
  *best_score = 0;
  *best_p0 = -inc;
  *best_p1 = -inc;
  *ops_bytes = 0;
  *rows = 0;
  if (q0[0] == delim || d0[0] == delim) return true;
  // row -1: the horizontal gap run from column 1 while >= -cutoff
  int k0;
  if (-gi < -cutoff) {
    k0 = 0;
  } else if (ge == 0) {
    k0 = 1 << 30;
  } else {
    const long long kk = ((long long)cutoff - gi) / ge + 1;
    k0 = kk > (1 << 30) ? (1 << 30) : (int)kk;
  }
  int col = find_delimiter_column(q0, inc, delim, 1, k0 > W ? W + 1 : k0);
  if (col > W) return false;
  for (int c = 1 + lane; c < col; c += 32) {
    const int s = -gi - (c - 1) * ge;
    band[c & wmask] = make_int2(s, s - gi);
  }
  if (lane == 0) band[0] = make_int2(0, -gi);
  int bs = 0, be;
  if (q0[(col - 1) * inc] != delim) {
    if (col + 1 > W) return false;
    if (lane == 0) band[col & wmask] = make_int2(kInitScore, kInitScore);
    be = col + 1;
  } else {
    be = col;
  }
  __syncwarp();

  int maxs = 0, mp0 = -inc, mp1 = -inc;
  uint64_t used = 0;
  uint64_t written = 0;  // end of the bytes the rows wrote
  uint32_t r = 0;
  for (;; ++r) {
    const int x = d0[(int)r * inc];
    if (x == delim) break;
    const int *mrow = sm + x * kMatrixStride;
    const int row_start = bs;
    uint8_t *row_ops = nullptr;
    if (STORE) {
      // a row's storage runs from its first band column to the next row's
      // band end: at most 2 W + 1 columns (the band, W wide, may move right
      // by up to W within the row), and the sentinel
      if (used + 2 * W + 2 > ops_cap || r >= rows_cap) return false;
      if (lane == 0) {
        row_meta[2 * r] = (uint32_t)used;
        row_meta[2 * r + 1] = (uint32_t)row_start;
      }
      row_ops = ops + used - row_start;
    }
    // column bs: vertical gap only
    const int2 st0 = band[bs & wmask];
    int diag = st0.x;
    const int nb0 = (maxs - st0.y > cutoff) ? kInitScore : st0.y;
    int F = nb0 - gi;   // horizontal gap without the reset at pruned cells
    int Fs = nb0 - gi;  // the reference's horizontal gap
    __syncwarp();
    if (lane == 0) {
      band[bs & wmask] = make_int2(nb0, st0.y - ge);
      if (STORE) row_ops[bs] = kTbGap0 + kTbExt0;
    }
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
      int prev = __shfl_up_sync(full, st.x, 1);
      if (lane == 0) prev = diag;
      const int sd = prev + mrow[qres];
      const int G = imax(sd, st.y);
      int P = active ? G - gi + (lane + 1) * ge : kNegBig;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int tv = __shfl_up_sync(full, P, o);
        if (lane >= o) P = imax(P, tv);
      }
      int Pex = __shfl_up_sync(full, P, 1);
      if (lane == 0) Pex = kNegBig;
      const int raw = imax(G, imax(F, Pex) - lane * ge);
      int R = active ? raw : kNegBig;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int tv = __shfl_up_sync(full, R, o);
        if (lane >= o) R = imax(R, tv);
      }
      const int Mrow = imax(M, R);
      const bool pruned = (Mrow - raw > cutoff);
      if (active) {
        const int nb = pruned ? kInitScore : raw;
        const int ng = pruned ? kInitScore : imax(raw - gi, st.y - ge);
        band[c & wmask] = make_int2(nb, ng);
      }
      const int nact = imin(32, be - cs);
      if (STORE) {
        // the reference's horizontal gap entering each cell: normalized
        // N(j) = F(j) + j ge obeys N(j + 1) = max(N(j), G(j) - gi + (j + 1) ge)
        // after a kept cell and restarts at kInitScore + (j + 1) ge after a
        // pruned one (a segment head)
        const bool head = active && pruned;
        int v = head ? kInitScore + (lane + 1) * ge : (active ? G - gi + (lane + 1) * ge : kNegBig);
        if (lane == 0 && !head) v = imax(v, Fs);
        bool seg = head;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int tv = __shfl_up_sync(full, v, o);
          const bool ts = __shfl_up_sync(full, seg, o);
          if (lane >= o) {
            if (!seg) v = imax(v, tv);
            seg = seg || ts;
          }
        }
        int Nin = __shfl_up_sync(full, v, 1);
        if (lane == 0) Nin = Fs;
        if (active && pruned) row_ops[c] = 0;
        if (active && !pruned) {
          const int Fb = Nin - lane * ge;
          int op = kTbSub, sc = sd;
          if (sc < st.y) {
            op = kTbGap0;
            sc = st.y;
          }
          if (sc < Fb) {
            op = kTbGap1;
            sc = Fb;
          }
          if (!(st.y - ge < sc - gi)) op += kTbExt0;
          if (!(Fb - ge < sc - gi)) op += kTbExt1;
          row_ops[c] = (uint8_t)op;
        }
        Fs = __shfl_sync(full, v, nact - 1) - nact * ge;
      }
      // new maximum: first column reaching the chunk maximum
      const int cm = __shfl_sync(full, R, 31);
      if (cm > M) {
        const unsigned hitm = __ballot_sync(full, active && raw == cm);
        const int l = __ffs(hitm) - 1;
        maxs = cm;
        mp0 = (cs + l - 1) * inc;
        mp1 = (int)r * inc;
      }
      const unsigned kept = __ballot_sync(full, active && !pruned);
      if (kept) {
        if (first_kept < 0) first_kept = cs + __ffs(kept) - 1;
        last_kept = cs + 31 - __clz(kept);
      }
      const int Plast = __shfl_sync(full, P, nact - 1);
      F = imax(F, Plast) - nact * ge;
      M = imax(M, cm);
      diag = __shfl_sync(full, st.x, 31);
    }
    __syncwarp();
    if (first_kept < 0) {  // every cell pruned: array_start + 1 == array_end
      written = used + (uint64_t)(be - row_start);
      ++r;
      break;
    }
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
        const long long kk = room / ge + 1;
        k = kk > (1 << 30) ? (1 << 30) : (int)kk;
      }
      if (k > 0) {
        const int lim = (be + k - bs > W) ? (W - (be - bs) + 1) : k;
        k = find_delimiter_column(q0, inc, delim, be, lim) - be;
        if (be + k - bs > W) return false;
        for (int j = lane; j < k; j += 32) {
          const int v = F - j * ge;
          band[(be + j) & wmask] = make_int2(v, v - gi);
          if (STORE) row_ops[be + j] = kTbGap0 + kTbExt0;
        }
        be += k;
      }
      edge_residue = q0[(be - 1) * inc] != delim;
    }
    if (edge_residue) {
      if (be + 1 - bs > W) return false;
      if (lane == 0) {
        band[be & wmask] = make_int2(kInitScore, kInitScore);
        if (STORE) row_ops[be] = 0;  // the sentinel
      }
      ++be;
    }
    used += (uint64_t)(be - row_start);
    written = used;
    __syncwarp();
  }
  *ops_bytes = used + (uint64_t)(t.len0 + 2);
  if (STORE) {
    // past the rows: zeros up to the storage the reference would keep
    if (*ops_bytes > ops_cap) return false;
    for (uint64_t j = written + lane; j < *ops_bytes; j += 32) ops[j] = 0;
    __syncwarp();
  }
  *rows = r;
  *best_score = maxs;
  *best_p0 = mp0;
  *best_p1 = mp1;
  return true;
}

}  // namespace

// Where BuildResult starts counting a side (src/aligner_build_results_thread.h:
// 110-160, src/aligner_common.h:275-340): the reverse side from the
// alignment start, the forward side from the hit.
__device__ __forceinline__ void tb_count_start(const TbArgs &a, uint64_t side, int p0, int p1,
                                               const uint8_t **qs, uint32_t *qp, uint32_t *dp) {
  const uint64_t slot = side >> 1;
  const uint32_t qi = (uint32_t)(slot / (uint64_t)a.max_results);
  const gzb_result r = a.results[slot];
  *qs = a.query + a.q_offsets[qi];
  if (side & 1) {
    *qp = r.hit_q;
    *dp = r.hit_d;
  } else {
    *qp = r.hit_q - 1 + (uint32_t)p0;
    *dp = r.hit_d - 1 + (uint32_t)p1;
  }
}

// PickOptimalPath (src/gapped_extender.cpp:473-531) from the best cell (p0,
// p1 in side coordinates) back to the origin, and BuildResult's counts over
// the path as AlignerBuildResultsThread::Run hands it over: the ops taken in
// reverse walk order, positions advancing from (qp, dp).  Op k of the walk
// is taken after the walk's later ops, so its positions are (qp, dp) plus
// the advances of the ops after it: the whole side's advance (p0 + 1 along
// the query, p1 + 1 along the database) less those of ops 0..k.  Row rr's
// op of column c sits at ops[meta[2 rr] + c - meta[2 rr + 1]]; a column
// left of the side's first row reads as 0, the byte the reference keeps
// before it.  Gap runs count as if the side followed a substitution.
__device__ TbStats tb_walk_stats(const uint8_t *ops, const uint32_t *meta, int inc, int p0,
                                 int p1, const uint8_t *qs, const uint8_t *db, uint32_t qp,
                                 uint32_t dp) {
  TbStats st;
  st.n = st.mismatches = st.openings = st.extensions = 0;
  int rr = p1 * inc, c0 = p0 * inc;
  const uint32_t qend = qp + (uint32_t)(c0 + 1), dend = dp + (uint32_t)(rr + 1);
  uint32_t qdone = 0, ddone = 0;  // advances of the ops walked so far
  int op = kTbSub;                // the DP's op state
  int last = -1;                  // the previous path op
  // a path op: its mismatch, and the gap count of the op walked before it
  // (taken right after this one)
  auto take = [&](int p) {
    if (p != kPathGap0) ++qdone;
    if (p != kPathGap1) ++ddone;
    if (p == kPathSub && qs[qend - qdone] != db[dend - ddone]) ++st.mismatches;
    if (last == kPathGap0 || last == kPathGap1) {
      if (p != last) ++st.openings; else ++st.extensions;
    }
    if (st.n == 0) st.last = (uint8_t)p;
    last = p;
    ++st.n;
  };
  while (rr >= 0 && c0 >= 0) {
    const long long at = (long long)meta[2 * rr] + (c0 + 1) - (long long)meta[2 * rr + 1];
    const int next = at >= 0 ? ops[at] : 0;
    if (op == kTbGap0) {
      op = next & 3;
      if (next & kTbExt0) op = kTbGap0;
    } else if (op == kTbGap1) {
      op = next & 3;
      if (next & kTbExt1) op = kTbGap1;
    } else {
      op = next & 3;
    }
    if (op == kTbGap0) {
      take(kPathGap0);
      --rr;
    } else if (op == kTbGap1) {
      take(kPathGap1);
      --c0;
    } else {
      take(kPathSub);
      --rr;
      --c0;
    }
  }
  for (; rr >= 0; --rr) take(kPathGap0);
  for (; c0 >= 0; --c0) take(kPathGap1);
  // the op walked last is taken first, after a substitution
  if (last == kPathGap0 || last == kPathGap1) ++st.openings;
  st.first = (uint8_t)(st.n ? last : kPathSub);
  if (st.n == 0) st.last = kPathSub;
  return st;
}

// One warp per side runs the DP with its ops and row table into the warp's
// own scratch (kTbScratchOps bytes, kTbScratchRows rows), where up to 32
// sides gather; then each lane walks one of them (PickOptimalPath and
// BuildResult's counts), the 32 walks in parallel, and the scratch is
// reused.  A side the warp cannot run exactly (X-drop >= 1024, a band wider
// than kTbWarpColumns) or whose storage outgrows an empty scratch is
// flagged in `redo` with its sizes left to the thread kernels; the others
// get zero sizes.
__global__ void __launch_bounds__(kTbWarpsPerBlock * 32, 4)
    tb_side_warp_kernel(TbArgs a, uint64_t n_sides, uint8_t *scratch, int32_t *side_score,
                        int32_t *side_p0, int32_t *side_p1, TbStats *stats, uint64_t *ops_bytes,
                        uint64_t *rows, uint8_t *redo) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  __shared__ int2 bands[kTbWarpsPerBlock][kTbWarpColumns];
  load_matrix(sm, a.matrix32, 32, 32);  // the 32 x 32 device matrix
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t *mine = scratch + (blockIdx.x * (uint64_t)kTbWarpsPerBlock + warp) * kTbScratchBytes;
  uint8_t *ops_arena = mine;
  uint32_t *meta_arena = reinterpret_cast<uint32_t *>(mine + kTbScratchOps);
  uint64_t ops_pos = 0;
  uint32_t meta_pos = 0, nacc = 0;
  // lane i: the i-th gathered side
  uint64_t my_side = 0, my_ops = 0;
  uint32_t my_meta = 0;
  int my_p0 = 0, my_p1 = 0, my_inc = 1;
  auto flush = [&]() {
    if ((uint32_t)lane < nacc) {
      const uint8_t *qs;
      uint32_t qp, dp;
      tb_count_start(a, my_side, my_p0, my_p1, &qs, &qp, &dp);
      stats[my_side] = tb_walk_stats(ops_arena + my_ops, meta_arena + 2 * (uint64_t)my_meta,
                                     my_inc, my_p0, my_p1, qs, a.db, qp, dp);
    }
    __syncwarp();
    ops_pos = 0;
    meta_pos = 0;
    nacc = 0;
  };
  for (uint64_t s = blockIdx.x * (uint64_t)kTbWarpsPerBlock + warp; s < n_sides;
       s += (uint64_t)gridDim.x * kTbWarpsPerBlock) {
    const TbSide t = side_of(a, s);
    bool ok = !t.active;
    if (t.active && a.cutoff < 1024) {
      for (int attempt = 0; attempt < 2 && !ok; ++attempt) {
        if (attempt == 1) {
          if (nacc == 0) break;  // outgrows even an empty scratch
          flush();
        }
        uint64_t nb;
        uint32_t nr;
        int sc, p0, p1;
        ok = tb_extend_warp<true>(a, sm, t, bands[warp], ops_arena + ops_pos,
                                  meta_arena + 2 * (uint64_t)meta_pos, kTbScratchOps - ops_pos,
                                  kTbScratchRows - meta_pos, &nb, &nr, &sc, &p0, &p1);
        if (ok) {
          if ((uint32_t)lane == nacc) {
            my_side = s;
            my_ops = ops_pos;
            my_meta = meta_pos;
            my_p0 = p0;
            my_p1 = p1;
            my_inc = t.inc;
            side_score[s] = sc;
            side_p0[s] = p0;
            side_p1[s] = p1;
          }
          ops_pos += nb;
          meta_pos += nr;
          if (++nacc == 32) flush();
        }
      }
    }
    if (lane == 0) {
      redo[s] = ok ? 0 : 1;
      ops_bytes[s] = 0;
      rows[s] = 0;
    }
    __syncwarp();
  }
  flush();
}

// per side flagged in `redo`: band columns (len0 + 2) for the scan
__global__ void tb_band_kernel(TbArgs a, uint64_t n_sides, const uint8_t *redo,
                               uint64_t *band_cols) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sides;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const TbSide t = side_of(a, s);
    band_cols[s] = (t.active && redo[s]) ? (uint64_t)t.len0 + 2 : 0;
  }
}

// the storage of the sides flagged in `redo` (one thread per side, the band
// in global memory)
__global__ void tb_count_kernel(TbArgs a, uint64_t n_sides, const uint64_t *band_off,
                                int2 *band, uint64_t *ops_bytes, uint64_t *rows,
                                const uint8_t *redo) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  load_matrix(sm, a.matrix32, 32, 32);  // the 32 x 32 device matrix
  __syncthreads();
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sides;
       s += (uint64_t)gridDim.x * blockDim.x) {
    if (!redo[s]) continue;
    const TbSide t = side_of(a, s);
    uint64_t nb = 0;
    uint32_t nr = 0;
    if (t.active) {
      int sc, p0, p1;
      tb_extend(a, sm, t, band + band_off[s], nullptr, nullptr, &nb, &nr, &sc, &p0, &p1);
    }
    ops_bytes[s] = t.active ? nb : 0;
    rows[s] = t.active ? nr : 0;
  }
}

// The flagged sides by one thread each: the DP with its ops (the band in
// global memory) into their own storage, then the walk and counts.
__global__ void tb_walk_kernel(TbArgs a, uint64_t n_sides, const uint64_t *band_off,
                               int2 *band, const uint64_t *ops_off, uint8_t *ops,
                               const uint64_t *rows_off, uint32_t *row_meta, int32_t *side_score,
                               int32_t *side_p0, int32_t *side_p1, TbStats *stats,
                               const uint8_t *redo) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  load_matrix(sm, a.matrix32, 32, 32);  // the 32 x 32 device matrix
  __syncthreads();
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sides;
       s += (uint64_t)gridDim.x * blockDim.x) {
    if (!redo[s]) continue;
    const TbSide t = side_of(a, s);
    if (!t.active) continue;
    uint8_t *sops = ops + ops_off[s];
    uint32_t *meta = row_meta + 2 * rows_off[s];
    uint64_t nb;
    uint32_t nr;
    int sc, p0, p1;
    tb_extend(a, sm, t, band + band_off[s], sops, meta, &nb, &nr, &sc, &p0, &p1);
    side_score[s] = sc;
    side_p0[s] = p0;
    side_p1[s] = p1;
    const uint8_t *qs;
    uint32_t qp, dp;
    tb_count_start(a, s, p0, p1, &qs, &qp, &dp);
    stats[s] = tb_walk_stats(sops, meta, t.inc, p0, p1, qs, a.db, qp, dp);
  }
}

// Joins the sides of each result as AlignerBuildResultsThread::Run does
// (src/aligner_build_results_thread.h:110-160): BuildResult
// (src/aligner_common.h:275-340) counts the reverse side's ops, then the
// forward side's, in one run, so a gap run that crosses from one side to
// the other is one opening.
__global__ void tb_combine_kernel(TbArgs a, uint64_t n_slots, const int32_t *side_score,
                                  const int32_t *side_p0, const int32_t *side_p1,
                                  const TbStats *stats, gzb_alignment *out) {
  for (uint64_t slot = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; slot < n_slots;
       slot += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t qi = (uint32_t)(slot / (uint64_t)a.max_results);
    const uint32_t k = (uint32_t)(slot % (uint64_t)a.max_results);
    if (qi >= a.nq || k >= a.counts[qi]) continue;
    const gzb_result r = a.results[slot];
    gzb_alignment o;
    o.chunk_id = r.chunk_id;
    o.subject_id = r.subject_id;
    o.score = r.score;
    o.hit_q = r.hit_q;
    o.hit_d = r.hit_d;
    o.start_q = r.start_q;
    o.start_d = r.start_d;
    o.end_q = r.end_q;
    o.end_d = r.end_d;
    o.alignment_length = o.mismatches = o.gap_openings = o.gap_extensions = 0;
    o.presearch_score = r.score;
    if (r.chunk_id == a.chunk_id) {
      const uint64_t sr = 2 * slot, sf = 2 * slot + 1;
      // AlignerBuildResultsThread::Run hands BuildResult the build step's
      // own score, start and end (src/aligner_build_results_thread.h:124-160)
      o.score = side_score[sr] + side_score[sf];
      o.start_q = r.hit_q - 1 + (uint32_t)side_p0[sr];
      o.start_d = r.hit_d - 1 + (uint32_t)side_p1[sr];
      o.end_q = r.hit_q + (uint32_t)side_p0[sf];
      o.end_d = r.hit_d + (uint32_t)side_p1[sf];
      const TbStats rv = stats[sr], fw = stats[sf];
      uint32_t op_n = rv.openings + fw.openings, ext_n = rv.extensions + fw.extensions;
      if (rv.n && fw.n && fw.first != kPathSub && fw.first == rv.last) {
        --op_n;  // the forward side's first gap continues the reverse side's last
        ++ext_n;
      }
      o.alignment_length = rv.n + fw.n;
      o.mismatches = rv.mismatches + fw.mismatches;
      o.gap_openings = op_n;
      o.gap_extensions = ext_n;
    }
    out[slot] = o;
  }
}

}  // namespace gzb
