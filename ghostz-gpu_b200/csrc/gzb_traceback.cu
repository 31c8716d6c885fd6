// gzb_traceback.cu -- alignment statistics of the merged results (the build
// results step): both sides of every result of the resident chunk are
// extended again with their edit path, and the path yields the figures
// AlignerCommon::BuildResult reports (alignment length, mismatches, gap
// openings and extensions).
//
// One thread per side.  Pass 1 runs the DP to size each side's op storage;
// pass 2 runs it again storing one op byte per kept cell, row by row, then
// walks the optimal path back from the best cell (PickOptimalPath); a last
// kernel joins the two sides per result in the reference's order.
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

}  // namespace

// per side: band columns (len0 + 2) for the scan
__global__ void tb_band_kernel(TbArgs a, uint64_t n_sides, uint64_t *band_cols) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sides;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const TbSide t = side_of(a, s);
    band_cols[s] = t.active ? (uint64_t)t.len0 + 2 : 0;
  }
}

// pass 1: op bytes and rows of every side
__global__ void tb_count_kernel(TbArgs a, uint64_t n_sides, const uint64_t *band_off,
                                int2 *band, uint64_t *ops_bytes, uint64_t *rows,
                                uint64_t *walk_cap) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  load_matrix(sm, a.matrix32, kMatrixStride, kMatrixStride);
  __syncthreads();
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sides;
       s += (uint64_t)gridDim.x * blockDim.x) {
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

// pass 2: the DP with its ops, then PickOptimalPath
// (src/gapped_extender.cpp:473-531); the path is written in walk order
// (from the best cell back to the origin).
__global__ void tb_walk_kernel(TbArgs a, uint64_t n_sides, const uint64_t *band_off,
                               int2 *band, const uint64_t *ops_off, uint8_t *ops,
                               const uint64_t *rows_off, uint32_t *row_meta,
                               const uint64_t *walk_off, uint8_t *walk, uint32_t *walk_n,
                               int32_t *side_score, int32_t *side_p0, int32_t *side_p1) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  load_matrix(sm, a.matrix32, kMatrixStride, kMatrixStride);
  __syncthreads();
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_sides;
       s += (uint64_t)gridDim.x * blockDim.x) {
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
