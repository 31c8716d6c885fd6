// gzb_karlin.cu -- per-query ungapped Karlin-Altschul statistics and the
// integer cutoffs derived from them, on the device (query preparation).
//
// For every query the reference builds (ProteinQuery / TranslatedDnaQuery,
// SetStaticalParameters) it takes the query's letter composition against
// the Robinson background (Statistics::CalculateUngappedKarlinParameters,
// src/statistics.cpp:205-229), solves lambda, H and K
// (ext/karlin/src/karlin.c, BlastKarlinBlkCalc), and turns them into the
// ungapped X-drop and the gapped-extension trigger
// (src/aligner_gpu.cpp:228-238, src/statistics.cpp:28-43).
//
// One warp per query, in two passes (buffers for 24 rounds of the K series,
// then for all 100 for the rare query that needs more).  The composition is
// counted by the whole warp; the
// score distribution's j-fold convolutions for K are spread over the lanes
// (each lane owns whole entries, so every entry is summed in the
// reference's order); every serial sum stays on lane 0 in the reference's
// order.  All arithmetic uses explicitly rounded operations (no fused
// multiply-add), so the float results agree with the reference's x86-64
// build bit for bit; exp, pow and log are CUDA's double-precision functions.
#include <cuda_runtime.h>

#include <cstdint>
#include <cmath>

#include "ghostz_b200.h"
#include "gzb_common.h"

namespace gzb {

namespace {

constexpr int kKarlinIterMax = 100;           // BLAST_KARLIN_K_ITER_MAX
// A first pass gives each warp convolution buffers for kFastIter rounds of
// the K series (the series usually ends after 10-15), so more warps fit on
// an SM; a query that needs more rounds is marked and redone by a second
// pass with buffers for all kKarlinIterMax rounds.
constexpr int kFastIter = 24, kFastWarps = 4;
constexpr int kFullWarps = 2;
constexpr int32_t kPending = INT32_MIN;       // cutoff of a query left to the second pass
constexpr int kMaxLetters = 32;
constexpr int kMaxRange = 31;                 // highest - lowest score
constexpr int kMaxRegular = 19;               // ARNDCQEGHILKMFPSTWYV

// Robinson & Robinson background, ARNDCQEGHILKMFPSTWYV order
// (src/statistics.cpp:154-176)
constexpr double kRobinson[20] = {78.05, 51.29, 44.87, 53.64, 19.25, 42.64, 62.95,
                                  73.77, 21.99, 51.42, 90.19, 57.44, 22.43, 38.56,
                                  52.03, 71.20, 58.41, 13.30, 32.16, 64.41};

struct KarlinArgs {
  double background[kMaxLetters];        // normalised letter probabilities
  // letter pairs grouped by score (score low + s owns pairs
  // [pair_begin[s], pair_begin[s + 1])), in (c1, c2) order within a group
  uint8_t pair_c1[kMaxLetters * kMaxLetters];
  uint8_t pair_c2[kMaxLetters * kMaxLetters];
  uint16_t pair_begin[kMaxRange + 2];
  int number_letters;                    // codes 0 .. number_letters-1
  int low, high;                         // score range of the matrix
  float ungapped_bits, trigger_bits, ln2;
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

__device__ bool range_bad(int lo, int hi) {
  return lo >= 0 || hi <= 0 || lo < -10000 || hi > 1000 || hi - lo > 11000;
}

__device__ long gcd_long(long a, long b) {
  long c;
  b = b < 0 ? -b : b;
  if (b > a) c = a, a = b, b = c;
  while (b != 0) {
    c = a % b;
    a = b;
    b = c;
  }
  return a;
}

// sum_i sp[i] exp(x i) the way the reference forms it: a running power
// from pow(exp(x), lo - 1), or exp(x i) per term once that underflows
__device__ double power_sum(const double *sp, int lo, int hi, double x) {
  const double x0 = exp(x);
  double x1 = pow(x0, (double)(lo - 1));
  double sum = 0.0;
  if (x1 > 0.0) {
    for (int i = lo; i <= hi; ++i) {
      x1 = dmul(x1, x0);
      sum = dadd(sum, dmul(sp[i], x1));
    }
  } else {
    for (int i = lo; i <= hi; ++i) sum = dadd(sum, dmul(sp[i], exp(dmul(x, (double)i))));
  }
  return sum;
}

// lambda by bisection (BlastKarlinLambdaBis)
__device__ double lambda_bisect(const double *sp, int lo, int hi) {
  if (range_bad(lo, hi)) return -1.0;
  double lambda = 0.0, up = 0.5;
  for (int guard = 0; guard < 2048; ++guard) {
    up = dmul(up, 2.0);
    if (power_sum(sp, lo, hi, up) >= 1.0) break;
    lambda = up;
  }
  for (int j = 0; j < 17; ++j) {
    const double mid = ddiv(dadd(lambda, up), 2.0);
    if (power_sum(sp, lo, hi, mid) > 1.0)
      up = mid;
    else
      lambda = mid;
  }
  return ddiv(dadd(lambda, up), 2.0);
}

// lambda by Newton-Raphson from 0.5 (BlastKarlinLambdaNR)
__device__ double lambda_newton(const double *sp, int lo, int hi) {
  if (range_bad(lo, hi)) return -1.0;
  double lambda = 0.5;
  for (int j = 0; j < 20; ++j) {
    double sum = -1.0, slope = 0.0;
    if (lambda < 0.01) break;
    const double x0 = exp(lambda);
    double x1 = pow(x0, (double)(lo - 1));
    if (x1 == 0.0) break;
    for (int i = lo; i <= hi; ++i) {
      x1 = dmul(x1, x0);
      const double t = dmul(sp[i], x1);
      sum = dadd(sum, t);
      slope = dadd(slope, dmul(t, (double)i));
    }
    const double step = ddiv(sum, slope);
    lambda = dsub(lambda, step);
    if (fabs(ddiv(step, lambda)) < 1.0e-5) {
      if (lambda > 1.0e-5) return lambda;
      break;
    }
  }
  return lambda_bisect(sp, lo, hi);
}

// relative entropy (BlastKarlinLtoH)
__device__ double entropy(const double *sp, int lo, int hi, double lambda) {
  if (lambda < 0.0 || range_bad(lo, hi)) return -1.0;
  const double etolam = exp(lambda);
  double etolami = pow(etolam, (double)(lo - 1)), av = 0.0;
  if (etolami > 0.0) {
    for (int s = lo; s <= hi; ++s) {
      etolami = dmul(etolami, etolam);
      av = dadd(av, dmul(dmul(sp[s], (double)s), etolami));
    }
  } else {
    for (int s = lo; s <= hi; ++s)
      av = dadd(av, dmul(dmul(sp[s], (double)s), exp(dmul(lambda, (double)s))));
  }
  return dmul(lambda, av);
}

// kIter: rounds of the K series the buffers hold.  kRetry: the second pass
// (only queries whose cutoff holds kPending).  The first pass runs eight
// blocks per SM (its grid), so it is bounded to the 64 registers that let
// all eight stay resident at once.
template <int kWarps, int kIter, bool kRetry>
__global__ void __launch_bounds__(kWarps * 32, kRetry ? 1 : 8)
    karlin_kernel(KarlinArgs a, const uint8_t *__restrict__ codes,
                  const uint64_t *__restrict__ offsets, const uint32_t *__restrict__ lengths,
                  uint32_t n, int32_t *__restrict__ cutoffs, int32_t *__restrict__ triggers,
                  float *__restrict__ karlin) {
  extern __shared__ double dist[];  // per warp: two convolution buffers
  __shared__ int count[kWarps][kMaxLetters];
  __shared__ double freq[kWarps][kMaxLetters];
  __shared__ double prob[kWarps][kMaxRange + 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int low = a.low, high = a.high, range = high - low;
  const int cap = kIter * range + 1;
  double *buf0 = dist + (size_t)w * 2 * cap, *buf1 = buf0 + cap;
  const int nl = a.number_letters;
  const uint32_t warps = gridDim.x * kWarps;
  for (uint32_t r = blockIdx.x * kWarps + w; r < n; r += warps) {
    if (kRetry && cutoffs[r] != kPending) continue;
    // composition of regular letters over the whole query
    count[w][lane] = 0;
    __syncwarp();
    const uint8_t *q = codes + offsets[r];
    const uint32_t len = lengths[r];
    for (uint32_t i = lane; i < len; i += 32) {
      const uint8_t c = q[i];
      if (c <= kMaxRegular) atomicAdd(&count[w][c], 1);
    }
    __syncwarp();
    // frequencies with a pseudo-count for absent letters, normalised
    if (lane < nl) freq[w][lane] = (double)count[w][lane] + (count[w][lane] < 1 ? 1.0 : 0.0);
    __syncwarp();
    double total = 0.0;
    if (lane == 0)
      for (int c = 0; c < nl; ++c) total = dadd(total, freq[w][c]);
    total = __shfl_sync(0xffffffffu, total, 0);
    if (lane < nl) freq[w][lane] = ddiv(freq[w][lane], total);
    __syncwarp();
    // score probabilities: lane s accumulates score low + s over its letter
    // pairs in the reference's (c1, c2) order
    if (lane <= range) {
      double acc = 0.0;
      for (int i = a.pair_begin[lane]; i < a.pair_begin[lane + 1]; ++i)
        acc = dadd(acc, dmul(freq[w][a.pair_c1[i]], a.background[a.pair_c2[i]]));
      prob[w][lane] = acc;
    }
    __syncwarp();
    if (lane == 0) {
      double s = 0.0;
      for (int i = 0; i <= range; ++i)
        if (prob[w][i] > 0.0) s = dadd(s, prob[w][i]);
      for (int i = 0; i <= range; ++i)
        if (prob[w][i] > 0.0) prob[w][i] = ddiv(prob[w][i], s);
    }
    __syncwarp();
    const double *sp = prob[w] - low;  // sp[score]
    const double *p = prob[w];         // p[u] = probability of score low + u
    // lambda and H on lane 0, rounded to float as BlastKarlinBlkCalc keeps them
    float l = 0.f, h = 0.f;
    if (lane == 0) {
      l = (float)lambda_newton(sp, low, high);
      h = (float)entropy(sp, low, high, (double)l);
    }
    l = __shfl_sync(0xffffffffu, l, 0);
    h = __shfl_sync(0xffffffffu, h, 0);
    // K (BlastKarlinLHtoK)
    const double lambda = (double)l, H = (double)h;
    double K = -1.0;
    bool pending = false;  // the series needs more rounds than the buffers hold
    if (lambda > 0.0 && H > 0.0) {
      const double av = ddiv(H, lambda);
      const double etolam = exp(lambda);
      if (low == -1 || high == 1) {
        K = dmul(av, dsub(1.0, ddiv(1.0, etolam)));
      } else {
        double sumlimit = 0.01;
        double sum = 1.0, oldsum = 1.0, oldsum2 = 1.0, Sum = 0.0;
        int lo = 0, hi = 0, j = 0;
        double *cur = buf0, *nxt = buf1;
        if (lane == 0) cur[0] = 1.0;
        __syncwarp();
        while (j < kIter && sum > sumlimit) {
          lo += low;
          hi += high;
          const int top = hi - lo;
          for (int k = lane; k <= top; k += 32) {
            const int first = range - (top - k) > 0 ? range - (top - k) : 0;
            const int last = k < range ? k : range;
            double s = 0.0;
            for (int u = first; u <= last; ++u) s = dadd(s, dmul(cur[k - u], p[u]));
            nxt[k] = s;
          }
          __syncwarp();
          double s = 0.0;
          if (lane == 0) {
            double etolami = pow(etolam, (double)(lo - 1));
            int i = lo, idx = 0;
            for (; i != 0; ++i, ++idx) {
              etolami = dmul(etolami, etolam);
              s = dadd(s, dmul(nxt[idx], etolami));
            }
            for (; i <= hi; ++i, ++idx) s = dadd(s, nxt[idx]);
          }
          s = __shfl_sync(0xffffffffu, s, 0);
          __syncwarp();
          oldsum2 = oldsum;
          oldsum = s;
          double *t = cur;
          cur = nxt;
          nxt = t;
          ++j;
          sum = ddiv(s, (double)j);
          Sum = dadd(Sum, sum);
        }
        const double ratio = ddiv(oldsum, oldsum2);
        if (kIter < kKarlinIterMax && j == kIter && sum > sumlimit) {
          pending = true;
        } else if (!(ratio >= dsub(1.0, dmul(sumlimit, 0.001)))) {
          sumlimit = dmul(sumlimit, 0.01);
          while (sum > sumlimit) {
            oldsum = dmul(oldsum, ratio);
            ++j;
            sum = ddiv(oldsum, (double)j);
            Sum = dadd(Sum, sum);
          }
          long delta = -low;
          for (int i = 1; i <= range && delta > 1; ++i)
            if (p[i] != 0.0) delta = gcd_long(delta, i);
          const double e2 = exp(dmul(-2.0, Sum));
          if (dmul((double)delta, etolam) > 0.05) {
            const double etolami = pow(etolam, (double)(-delta));
            K = ddiv(dmul((double)delta, e2), dmul(av, dsub(1.0, etolami)));
          } else {
            K = ddiv(dmul((double)(-delta), e2),
                     dmul(av, dsub(exp(dmul((double)(-delta), lambda)), 1.0)));
          }
        }
      }
    }
    if (lane == 0 && pending) cutoffs[r] = kPending;
    if (lane == 0 && !pending) {
      const float k = (float)K;
      // NormalizedCutoff2NominalCutoff and Normalized2Nominal in float; ln K
      // is the float nearest the exact logarithm
      const float c = __fdiv_rn(__fmul_rn(a.ungapped_bits, a.ln2), l);
      const float t =
          __fdiv_rn(__fadd_rn(__fmul_rn(a.trigger_bits, a.ln2), (float)log((double)k)), l);
      cutoffs[r] = (int32_t)floorf(c);
      triggers[r] = (int32_t)floorf(t);
      if (karlin) {
        karlin[3 * (size_t)r] = l;
        karlin[3 * (size_t)r + 1] = k;
        karlin[3 * (size_t)r + 2] = h;
      }
    }
    __syncwarp();
  }
}

}  // namespace

}  // namespace gzb

extern "C" int gzb_query_karlin_cutoffs(const uint8_t *d_codes, const uint64_t *d_offsets,
                                        const uint32_t *d_lengths, uint32_t number_queries,
                                        const int32_t *score_matrix, uint32_t number_letters,
                                        float ungapped_bits, float trigger_bits,
                                        int32_t *d_cutoffs, int32_t *d_triggers,
                                        float *d_karlin, void *stream) {
  using namespace gzb;
  GZB_CHECK(score_matrix, GZB_ERR_INVALID, "gzb_query_karlin_cutoffs: null score matrix");
  GZB_CHECK(number_letters > kMaxRegular && number_letters <= kMaxLetters, GZB_ERR_INVALID,
            "gzb_query_karlin_cutoffs: %u letters (protein alphabets of 20..32 codes)",
            number_letters);
  KarlinArgs a;
  int lo = score_matrix[0], hi = score_matrix[0];
  for (uint32_t i = 0; i < number_letters * number_letters; ++i) {
    lo = score_matrix[i] < lo ? score_matrix[i] : lo;
    hi = score_matrix[i] > hi ? score_matrix[i] : hi;
  }
  GZB_CHECK(lo < 0 && hi > 0, GZB_ERR_INVALID,
            "gzb_query_karlin_cutoffs: scores must span negative and positive values");
  GZB_CHECK(hi - lo <= kMaxRange, GZB_ERR_OVERFLOW,
            "gzb_query_karlin_cutoffs: score range %d exceeds %d", hi - lo, kMaxRange);
  int at = 0;
  for (int s = 0; s <= hi - lo; ++s) {
    a.pair_begin[s] = (uint16_t)at;
    for (uint32_t c1 = 0; c1 < number_letters; ++c1)
      for (uint32_t c2 = 0; c2 < number_letters; ++c2)
        if (score_matrix[c1 * number_letters + c2] == lo + s) {
          a.pair_c1[at] = (uint8_t)c1;
          a.pair_c2[at] = (uint8_t)c2;
          ++at;
        }
  }
  a.pair_begin[hi - lo + 1] = (uint16_t)at;
  // background, normalised in the reference's order (Statistics::Statistics)
  double sum = 0.0;
  for (int c = 0; c < kMaxLetters; ++c) a.background[c] = c < 20 ? kRobinson[c] : 0.0;
  for (uint32_t c = 0; c < number_letters; ++c) sum += a.background[c];
  for (uint32_t c = 0; c < number_letters; ++c) a.background[c] /= sum;
  a.number_letters = (int)number_letters;
  a.low = lo;
  a.high = hi;
  a.ungapped_bits = ungapped_bits;
  a.trigger_bits = trigger_bits;
  a.ln2 = (float)std::log(2.0);
  if (number_queries == 0) return GZB_OK;
  GZB_CHECK(d_codes && d_offsets && d_lengths && d_cutoffs && d_triggers, GZB_ERR_INVALID,
            "gzb_query_karlin_cutoffs: null buffer");
  int device = 0, sms = 148;
  GZB_CUDA(cudaGetDevice(&device));
  GZB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int range = hi - lo;
  // pass 1: buffers for kFastIter rounds; pass 2: the queries it left
  const size_t smem_fast = (size_t)kFastWarps * 2 * (kFastIter * range + 1) * sizeof(double);
  const size_t smem_full = (size_t)kFullWarps * 2 * (kKarlinIterMax * range + 1) * sizeof(double);
  auto fast = karlin_kernel<kFastWarps, kFastIter, false>;
  auto full = karlin_kernel<kFullWarps, kKarlinIterMax, true>;
  GZB_CUDA(cudaFuncSetAttribute(fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fast));
  GZB_CUDA(cudaFuncSetAttribute(full, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_full));
  const uint64_t want_fast = (number_queries + kFastWarps - 1) / kFastWarps;
  const uint64_t most_fast = (uint64_t)sms * 8;
  fast<<<(unsigned)(want_fast < most_fast ? want_fast : most_fast), kFastWarps * 32, smem_fast,
         (cudaStream_t)stream>>>(a, d_codes, d_offsets, d_lengths, number_queries, d_cutoffs,
                                 d_triggers, d_karlin);
  GZB_CUDA(cudaGetLastError());
  const uint64_t want_full = (number_queries + kFullWarps - 1) / kFullWarps;
  const uint64_t most_full = (uint64_t)sms * 4;
  full<<<(unsigned)(want_full < most_full ? want_full : most_full), kFullWarps * 32, smem_full,
         (cudaStream_t)stream>>>(a, d_codes, d_offsets, d_lengths, number_queries, d_cutoffs,
                                 d_triggers, d_karlin);
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}
