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

// Features of one extension starting at q0/d0 (query/database), stepping
// by inc: the ungapped X-drop score along the diagonal, the number of
// residue pairs it examined, positives and identities among the first 16
// pairs, remaining query / subject residues in the extension direction and
// the direction itself.
__device__ __forceinline__ void extension_features(const uint8_t *q0, const uint8_t *d0, int inc,
                                                   int delim, const int *matrix32, int cutoff,
                                                   uint32_t len0, uint32_t len1, bool reverse,
                                                   float *f) {
  int best = 0, run = 0, pos = 0, steps = 0, positives = 0, identities = 0;
  for (int k = 0; k < 4096; ++k) {
    const int a = q0[pos], b = d0[pos];
    if (a == delim || b == delim) break;
    const int sc = matrix32[b * 32 + a];
    if (k < 16) {
      positives += sc > 0;
      identities += a == b;
    }
    run += sc;
    pos += inc;
    ++steps;
    if (run > 0) {
      best += run;
      run = 0;
    } else if (run <= -cutoff) {
      break;
    }
  }
  f[0] = best * (1.0f / 32.0f);
  f[1] = log2f(1.0f + (float)len0) * 0.125f;
  f[2] = log2f(1.0f + (float)len1) * 0.125f;
  f[3] = reverse ? 1.0f : 0.0f;
  f[4] = positives * (1.0f / 16.0f);
  f[5] = identities * (1.0f / 16.0f);
  f[6] = log2f(1.0f + (float)steps) * 0.125f;
  f[7] = log2f(1.0f + (float)(len0 < len1 ? len0 : len1)) * 0.125f;
}

}  // namespace gzb
