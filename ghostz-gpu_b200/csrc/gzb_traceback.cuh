// gzb_traceback.cuh -- kernels of the build results step (gzb_traceback.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ghostz_b200.h"

namespace gzb {

// Inputs shared by the build results kernels.  Sides are numbered
// 2 * slot + {0 reverse, 1 forward}, slot = query * max_results + rank.
struct TbArgs {
  const uint8_t *query;  // concatenated queries (query id q starts at q_offsets[q])
  const uint8_t *db;     // the resident chunk
  const int32_t *matrix32;
  const uint32_t *q_offsets, *q_lengths;
  const gzb_result *results;
  const uint32_t *counts;
  uint32_t nq;
  int max_results;
  int32_t chunk_id;
  int delim, gap_open, gap_ext, cutoff;
};

// One side's counts for BuildResult, its ops taken in reverse walk order:
// ops, mismatches, gap openings and extensions (as if the side followed a
// substitution), and the first and last op taken (kPath* codes).
struct TbStats {
  uint32_t n, mismatches, openings, extensions;
  uint8_t first, last;
};

// each warp of tb_side_warp_kernel gathers up to 32 sides' ops
// (kTbScratchOps bytes) and row tables (kTbScratchRows rows) in its own
// kTbScratchBytes of scratch before walking them
constexpr uint64_t kTbScratchOps = 256 * 1024;
constexpr uint32_t kTbScratchRows = 8192;
constexpr uint64_t kTbScratchBytes = kTbScratchOps + 8ull * kTbScratchRows;

__global__ void tb_band_kernel(TbArgs a, uint64_t n_sides, const uint8_t *redo,
                               uint64_t *band_cols);
// warps per block of the one-warp-per-side kernel
constexpr int kTbWarpBlock = 8 * 32;
__global__ void tb_side_warp_kernel(TbArgs a, uint64_t n_sides, uint8_t *scratch,
                                    int32_t *side_score, int32_t *side_p0, int32_t *side_p1,
                                    TbStats *stats, uint64_t *ops_bytes, uint64_t *rows,
                                    uint8_t *redo);
__global__ void tb_count_kernel(TbArgs a, uint64_t n_sides, const uint64_t *band_off,
                                int2 *band, uint64_t *ops_bytes, uint64_t *rows,
                                const uint8_t *redo);
__global__ void tb_walk_kernel(TbArgs a, uint64_t n_sides, const uint64_t *band_off,
                               int2 *band, const uint64_t *ops_off, uint8_t *ops,
                               const uint64_t *rows_off, uint32_t *row_meta, int32_t *side_score,
                               int32_t *side_p0, int32_t *side_p1, TbStats *stats,
                               const uint8_t *redo);
__global__ void tb_combine_kernel(TbArgs a, uint64_t n_slots, const int32_t *side_score,
                                  const int32_t *side_p0, const int32_t *side_p1,
                                  const TbStats *stats, gzb_alignment *out);

}  // namespace gzb
