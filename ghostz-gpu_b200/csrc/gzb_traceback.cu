// gzb_traceback.cu -- alignment statistics of the merged results (the build
// results step): both sides of every result of the resident chunk are
// extended again with their edit path, and the path yields the figures
// AlignerCommon::BuildResult reports (alignment length, mismatches, gap
// openings and extensions).
//
// Pass 1 runs the DP to size each side's op storage; pass 2 runs it again
// storing one op byte per kept cell, row by row; then each side's optimal
// path is walked back from the best cell (PickOptimalPath); a last kernel
// joins the two sides per result in the reference's order.
//
// Both DP passes give one warp to a side: the warp evaluates 32 consecutive
// columns of a row at once, with the presearch's warp DP
// (gapped_extend_warp in gzb_kernels.cuh: band edges and stored values
// exact for X-drops below 1024).  A kept cell's edit op also needs the
// reference's horizontal-gap value *with* its reset to kInitScore at pruned
// cells (src/gapped_extender.cpp:428-446); once a chunk's pruned flags are
// known that value is a segmented max-plus scan whose segments start after
// the pruned cells.  Sides whose band outgrows the warp's circular buffer,
// or whose X-drop is 1024 or more, are flagged and run by one thread each
// with the band in global memory (the serial form of the same DP).
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
// STORE it also writes the ops and row table as tb_extend does.  Returns
// false when the band outgrows kTbWarpColumns (outputs then meaningless).
template <bool STORE>
__device__ bool tb_extend_warp(const TbArgs &a, const int *sm, const TbSide &t, int2 *band,
                               uint8_t *ops, uint32_t *row_meta, uint64_t *ops_bytes,
                               uint32_t *rows, int *best_score, int *best_p0, int *best_p1) {
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
  uint32_t r = 0;
  for (;; ++r) {
    const int x = d0[(int)r * inc];
    if (x == delim) break;
    const int *mrow = sm + x * kMatrixStride;
    const int row_start = bs;
    uint8_t *row_ops = nullptr;
    if (STORE) {
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
      if (lane == 0) band[be & wmask] = make_int2(kInitScore, kInitScore);
      ++be;
    }
    used += (uint64_t)(be - row_start);
    __syncwarp();
  }
  *ops_bytes = used + (uint64_t)(t.len0 + 2);
  *rows = r;
  *best_score = maxs;
  *best_p0 = mp0;
  *best_p1 = mp1;
  return true;
}

}  // namespace

// pass 1 by one warp per side; a side the warp cannot run exactly is
// flagged in `redo` for tb_count_kernel
__global__ void __launch_bounds__(kTbWarpsPerBlock * 32)
    tb_count_warp_kernel(TbArgs a, uint64_t n_sides, uint64_t *ops_bytes, uint64_t *rows,
                         uint64_t *walk_cap, uint8_t *redo) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  __shared__ int2 bands[kTbWarpsPerBlock][kTbWarpColumns];
  load_matrix(sm, a.matrix32, 32, 32);  // the 32 x 32 device matrix
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t s = blockIdx.x * (uint64_t)kTbWarpsPerBlock + warp; s < n_sides;
       s += (uint64_t)gridDim.x * kTbWarpsPerBlock) {
    const TbSide t = side_of(a, s);
    bool ok = true;
    uint64_t nb = 0;
    uint32_t nr = 0;
    if (t.active) {
      int sc, p0, p1;
      ok = a.cutoff < 1024 &&
           tb_extend_warp<false>(a, sm, t, bands[warp], nullptr, nullptr, &nb, &nr, &sc, &p0,
                                 &p1);
    }
    if (lane == 0) {
      redo[s] = ok ? 0 : 1;
      ops_bytes[s] = t.active ? nb : 0;
      rows[s] = t.active ? nr : 0;
      walk_cap[s] = t.active ? (uint64_t)nr + t.len0 + 2 : 0;
    }
    __syncwarp();
  }
}

// pass 2 by one warp per side for the sides pass 1 ran by warp: the DP with
// its ops and row table, and the side's best score and positions
__global__ void __launch_bounds__(kTbWarpsPerBlock * 32)
    tb_store_warp_kernel(TbArgs a, uint64_t n_sides, const uint64_t *ops_off, uint8_t *ops,
                         const uint64_t *rows_off, uint32_t *row_meta, int32_t *side_score,
                         int32_t *side_p0, int32_t *side_p1, const uint8_t *redo) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  __shared__ int2 bands[kTbWarpsPerBlock][kTbWarpColumns];
  load_matrix(sm, a.matrix32, 32, 32);  // the 32 x 32 device matrix
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t s = blockIdx.x * (uint64_t)kTbWarpsPerBlock + warp; s < n_sides;
       s += (uint64_t)gridDim.x * kTbWarpsPerBlock) {
    if (redo[s]) continue;
    const TbSide t = side_of(a, s);
    if (!t.active) continue;
    uint64_t nb;
    uint32_t nr;
    int sc, p0, p1;
    tb_extend_warp<true>(a, sm, t, bands[warp], ops + ops_off[s], row_meta + 2 * rows_off[s],
                         &nb, &nr, &sc, &p0, &p1);
    if (lane == 0) {
      side_score[s] = sc;
      side_p0[s] = p0;
      side_p1[s] = p1;
    }
    __syncwarp();
  }
}

// per side: band columns (len0 + 2) for the scan
__global__ void tb_band_kernel(TbArgs a, uint64_t n_sides, uint64_t *band_cols) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sides;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const TbSide t = side_of(a, s);
    band_cols[s] = t.active ? (uint64_t)t.len0 + 2 : 0;
  }
}

// pass 1 by one thread per side for the sides flagged in `redo`, the band in
// global memory
__global__ void tb_count_kernel(TbArgs a, uint64_t n_sides, const uint64_t *band_off,
                                int2 *band, uint64_t *ops_bytes, uint64_t *rows,
                                uint64_t *walk_cap, const uint8_t *redo) {
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
    // the path has at most one op per row plus one per seq0 residue
    walk_cap[s] = t.active ? (uint64_t)nr + t.len0 + 2 : 0;
  }
}

// pass 2 for the flagged sides (the DP with its ops by one thread, the band
// in global memory), then PickOptimalPath (src/gapped_extender.cpp:473-531)
// for every side; the path is written in walk order (from the best cell
// back to the origin).
__global__ void tb_walk_kernel(TbArgs a, uint64_t n_sides, const uint64_t *band_off,
                               int2 *band, const uint64_t *ops_off, uint8_t *ops,
                               const uint64_t *rows_off, uint32_t *row_meta,
                               const uint64_t *walk_off, uint8_t *walk, uint32_t *walk_n,
                               int32_t *side_score, int32_t *side_p0, int32_t *side_p1,
                               const uint8_t *redo) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  load_matrix(sm, a.matrix32, 32, 32);  // the 32 x 32 device matrix
  __syncthreads();
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sides;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const TbSide t = side_of(a, s);
    if (!t.active) continue;
    uint8_t *sops = ops + ops_off[s];
    uint32_t *meta = row_meta + 2 * rows_off[s];
    int p0, p1;
    if (redo[s]) {
      uint64_t nb;
      uint32_t nr;
      int sc;
      tb_extend(a, sm, t, band + band_off[s], sops, meta, &nb, &nr, &sc, &p0, &p1);
      side_score[s] = sc;
      side_p0[s] = p0;
      side_p1[s] = p1;
    } else {
      p0 = side_p0[s];
      p1 = side_p1[s];
    }
    uint8_t *path = walk + walk_off[s];
    uint32_t m = 0;
    {
      int op = kTbSub;
      int rr = p1 * t.inc, c0 = p0 * t.inc;
      while (rr >= 0 && c0 >= 0) {
        // op of column c0 + 1 of row rr; a column left of the side's first
        // row reads as 0, the byte the reference keeps before its first row
        const long long at = (long long)meta[2 * rr] + (c0 + 1) - (long long)meta[2 * rr + 1];
        const int next = at >= 0 ? sops[at] : 0;
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
          path[m++] = kPathGap0;
          --rr;
        } else if (op == kTbGap1) {
          path[m++] = kPathGap1;
          --c0;
        } else {
          path[m++] = kPathSub;
          --rr;
          --c0;
        }
      }
      for (; rr >= 0; --rr) path[m++] = kPathGap0;
      for (; c0 >= 0; --c0) path[m++] = kPathGap1;
    }
    walk_n[s] = m;
  }
}

// Joins the sides of each result as AlignerBuildResultsThread::Run does
// (src/aligner_build_results_thread.h:110-160): the reverse side's edit
// blocks reversed, then the forward side's, where both sides' blocks are
// their paths in walk order reversed; then AlignerCommon::BuildResult
// (src/aligner_common.h:275-340) counts from the alignment start.
__global__ void tb_combine_kernel(TbArgs a, uint64_t n_slots, const uint64_t *walk_off,
                                  const uint8_t *walk, const uint32_t *walk_n,
                                  const int32_t *side_score, const int32_t *side_p0,
                                  const int32_t *side_p1, gzb_alignment *out) {
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
      const uint8_t *qs = a.query + a.q_offsets[qi];
      // AlignerBuildResultsThread::Run hands BuildResult the build step's
      // own score, start and end (src/aligner_build_results_thread.h:124-160)
      o.score = side_score[sr] + side_score[sf];
      o.start_q = r.hit_q - 1 + (uint32_t)side_p0[sr];
      o.start_d = r.hit_d - 1 + (uint32_t)side_p1[sr];
      o.end_q = r.hit_q + (uint32_t)side_p0[sf];
      o.end_d = r.hit_d + (uint32_t)side_p1[sf];
      uint32_t qp = r.hit_q - 1 + (uint32_t)side_p0[sr];
      uint32_t dp = r.hit_d - 1 + (uint32_t)side_p1[sr];
      uint32_t mm = 0, op_n = 0, ext_n = 0;
      int prev = kPathSub;
      const uint32_t nr = walk_n[sr], nf = walk_n[sf];
      const uint8_t *pr = walk + walk_off[sr], *pf = walk + walk_off[sf];
      for (uint32_t i = 0; i < nr + nf; ++i) {
        const int op = i < nr ? pr[nr - 1 - i] : pf[nr + nf - 1 - i];
        if (op == kPathSub) {
          if (qs[qp] != a.db[dp]) ++mm;
          ++qp;
          ++dp;
        } else if (op == kPathGap0) {
          if (prev != kPathGap0) ++op_n; else ++ext_n;
          ++dp;
        } else {
          if (prev != kPathGap1) ++op_n; else ++ext_n;
          ++qp;
        }
        prev = op;
      }
      o.alignment_length = nr + nf;
      o.mismatches = mm;
      o.gap_openings = op_n;
      o.gap_extensions = ext_n;
    }
    out[slot] = o;
  }
}

}  // namespace gzb
