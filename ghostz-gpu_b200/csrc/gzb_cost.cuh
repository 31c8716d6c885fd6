// gzb_cost.cuh -- cost model of the gapped stage: per-extension features and
// a small MLP (8 -> 32 -> 32 -> 1, ReLU) that predicts log2(1 + DP cells).
//
// The model only reorders work: the batched schedule runs extensions
// longest-predicted first so that the 32 extensions a warp takes together
// have similar cost.  Every extension is still computed by the same exact
// kernel, so results do not depend on the model.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace gzb {

constexpr int kFeat = 8;
constexpr int kHid = 32;
// parameter layout: W1[kHid][kFeat], b1[kHid], W2[kHid][kHid], b2[kHid],
// W3[kHid], b3
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHid * kFeat;
constexpr int kOffW2 = kOffB1 + kHid;
constexpr int kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid;
constexpr int kOffB3 = kOffW3 + kHid;
constexpr int kParams = kOffB3 + 1;  // 1377

// Ungapped X-drop walk along the diagonal from q0/d0 (query/database),
// stepping by inc, as the ungapped extension scores it: the best score and
// the number of residue pairs examined before the drop (or a delimiter).
__device__ __forceinline__ void diagonal_walk(const uint8_t *q0, const uint8_t *d0, int inc,
                                              int delim, const int *matrix32, int cutoff,
                                              int *best_out, int *steps_out) {
  int best = 0, run = 0, pos = 0, steps = 0;
  for (int k = 0; k < 4096; ++k) {
    const int a = q0[pos], b = d0[pos];
    if (a == delim || b == delim) break;
    run += matrix32[b * 32 + a];
    pos += inc;
    ++steps;
    if (run > 0) {
      best += run;
      run = 0;
    } else if (run <= -cutoff) {
      break;
    }
  }
  *best_out = best;
  *steps_out = steps;
}

// Features of one extension of a chained hit:
//  f0 the hit's ungapped score (both directions' diagonal walks),
//  f1/f2 remaining query / subject residues in the extension direction,
//  f3 the direction, f4 this direction's walk score, f5 chained hits of the
//  same query within 256 database residues (a homologous region yields
//  many), f6 the walk length (local similarity of the residues along the
//  diagonal), f7 the shorter remaining length.  Lengths and counts enter as
//  log2(1 + x) / 8, scores as x / 32.
__device__ __forceinline__ void extension_features(int best, int pair_best, int steps,
                                                   uint32_t len0, uint32_t len1, bool reverse,
                                                   uint32_t neighbours, float *f) {
  f[0] = pair_best * (1.0f / 32.0f);
  f[1] = log2f(1.0f + (float)len0) * 0.125f;
  f[2] = log2f(1.0f + (float)len1) * 0.125f;
  f[3] = reverse ? 1.0f : 0.0f;
  f[4] = best * (1.0f / 32.0f);
  f[5] = log2f(1.0f + (float)neighbours) * 0.125f;
  f[6] = log2f(1.0f + (float)steps) * 0.125f;
  f[7] = log2f(1.0f + (float)(len0 < len1 ? len0 : len1)) * 0.125f;
}

}  // namespace gzb
