// gzb_seg.cu -- SEG low-complexity masking of query sequences on the device
// (query preparation with the aln default filter on, -F T).
//
// The masking is the reference's vendored SEG (ext/seg/src/seg.cpp) as
// SequenceSegFilter applies it (src/sequence_seg_filter.cpp:17-23):
//   * window 12; the entropy H(i) of position i is that of the 12 letters
//     starting at i, and past length - 12 that of the last full window;
//   * a position with H <= 2.2 bits seeds a segment, which grows left and
//     right while H <= 2.5 (left no further than the end of the previous
//     segment), is trimmed to its least probable sub-window (lengths down
//     to 100 below the segment's), and the part left of the trimmed
//     segment is searched again on its own;
//   * segments are masked to the unknown letter; a sequence shorter than
//     the window is not masked and the caller's fallback applies (unknown
//     letters for a translated frame, src/translated_dna_query.cpp:59-65;
//     a body of code 0 for a protein query, src/protein_query.cpp:39-49).
// Only the 20 standard amino acids count towards compositions.
//
// Two passes over the sequences (frames of translated queries or bodies of
// protein queries), in place.  Pass 1, one thread per frame (a warp per
// protein, its windows split over the lanes), only computes the window
// entropies; a sequence with no window at or below the
// low cut (most of them) is done, the others are marked.  Pass 2, one warp
// per marked sequence, runs the whole search: masked positions get bit 6
// set while it runs (so later windows still see the letters) and become the
// unknown code at the end; the trimming search, the costly part, is split
// over the lanes.  The left recursion runs on an explicit stack of at most
// kSegStack frames; deeper nesting (which the trimming rule bounds well
// below that) is counted in the status word and leaves the sequence
// unmasked.  All floating point is adds and subtracts of tables computed on
// the host with the host's log (plus one multiply per window), in the
// reference's order, so every comparison matches.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "ghostz_b200.h"
#include "gzb_common.h"

namespace gzb {

namespace {

constexpr int kSegWindow = 12;
constexpr double kSegLowCut = 2.2;
constexpr double kSegHighCut = 2.5;
constexpr int kSegMaxTrim = 100;
constexpr int kSegStack = 96;
constexpr int kSegMaxLength = 65535;      // ln(n!) table covers n <= this
constexpr uint8_t kMaskBit = 64;
constexpr uint8_t kUnknownCode = 24;      // X
constexpr int kSegBlock = 128;
// window entropies a warp of the search pass keeps in shared memory (the
// windows of sequences up to `cache` + 11 residues): 1024 for the short
// frames of translated reads (four warps a block), 4096 for proteins (two)
constexpr int kSegCacheFrames = 1024;
constexpr int kSegCacheProteins = 4096;

// ln(n!) rounded to 6 decimals (the precision of the reference's table)
__device__ double g_seg_ln_fact[kSegMaxLength + 1];

struct SegArgs {
  double entropy12[kSegWindow + 1];                 // windows of 12 letters
  double log_ratio[kSegWindow][kSegWindow + 1];     // log(v * (1/total))
  double ln2, ln20;
};

// code of an amino acid SEG counts: the 20 standard letters (codes 0-19);
// bit 5 marks a letter the caller wants ignored, bit 6 a masked position
__device__ __forceinline__ int seg_class(uint8_t v) {
  const int c = v & 63;
  return c < 20 ? c : -1;
}

// counts of the letters in s[0..n), decreasing, 0-terminated
__device__ void seg_state(const uint8_t *s, int n, int *comp, int *state) {
  for (int k = 0; k < 20; ++k) comp[k] = 0;
  for (int i = 0; i < n; ++i) {
    const int k = seg_class(s[i]);
    if (k >= 0) ++comp[k];
  }
  int m = 0;
  for (int k = 0; k < 20; ++k)
    if (comp[k]) state[m++] = comp[k];
  for (int a = 1; a < m; ++a)
    for (int b = a; b > 0 && state[b - 1] < state[b]; --b) {
      const int t = state[b];
      state[b] = state[b - 1];
      state[b - 1] = t;
    }
  for (int k = m; k <= 20; ++k) state[k] = 0;
}

// one more of a letter whose count was c: the first entry equal to c grows
__device__ void state_grow(int *state, int c) {
  for (int i = 0; i < 20; ++i)
    if (state[i] == c) {
      ++state[i];
      return;
    }
}

// one fewer of a letter whose count was c: the last entry equal to c shrinks
__device__ void state_shrink(int *state, int c) {
  for (int i = 0; state[i] != 0; ++i)
    if (state[i] == c && state[i + 1] < c) {
      --state[i];
      return;
    }
}

__device__ double seg_entropy(const SegArgs &a, const int *state) {
  int total = 0, m = 0;
  for (; m < 20 && state[m]; ++m) total += state[m];
  double ent = 0.0;
  if (total == kSegWindow) {
    for (int i = 0; i < m; ++i) ent = __dadd_rn(ent, a.entropy12[state[i]]);
    return ent;
  }
  if (total == 0) return 0.0;
  const double r = __ddiv_rn(1.0, (double)total);
  for (int i = 0; i < m; ++i)
    ent = __dadd_rn(ent, __dmul_rn((double)state[i], a.log_ratio[total][state[i]]));
  return __ddiv_rn(__dmul_rn(-ent, r), a.ln2);
}

__device__ double seg_h(const SegArgs &a, const uint8_t *s, int n, int i) {
  int comp[20], state[21];
  const int start = i < n - kSegWindow ? i : n - kSegWindow;
  seg_state(s + start, kSegWindow, comp, state);
  return seg_entropy(a, state);
}

// ln probability of a window's composition (LnAss + LnPerm - n ln 20)
__device__ double seg_probability(const SegArgs &a, const int *state, int total) {
  const double *T = g_seg_ln_fact;
  double ass = T[20];
  if (state[0] != 0) {
    int left = 20, run = 1, prev = state[0];
    for (int i = 1; i < 20; ++i) {
      const int v = state[i];
      if (v == prev) {
        ++run;
      } else {
        left -= run;
        ass = __dsub_rn(ass, T[run]);
        if (v == 0) {
          run = left;
          break;
        }
        run = 1;
      }
      prev = v;
    }
    ass = __dsub_rn(ass, T[run]);
  }
  double perm = T[total];
  for (int i = 0; i < 20 && state[i] != 0; ++i) perm = __dsub_rn(perm, T[state[i]]);
  return __dsub_rn(__dadd_rn(ass, perm), __dmul_rn((double)total, a.ln20));
}

// The least probable sub-window of s[0..n) over lengths n .. max(1, n-100)+1
// (the reference's first minimum in the order length descending, start
// ascending).  The whole warp calls it with the same arguments: lane l
// takes the lengths n - l, n - l - 32, ..., slides each over s with the
// reference's count updates, and the warp keeps the smallest (probability,
// order) pair, which is the serial search's first minimum.
__device__ void seg_trim_warp(const SegArgs &a, const uint8_t *s, int n, int *left, int *right,
                              int lane) {
  const int min_length = n - kSegMaxTrim > 1 ? n - kSegMaxTrim : 1;
  const int lens = n - min_length;  // lengths n, n-1, ..., min_length+1
  double best = 1.0;
  uint64_t best_at = ~0ull;         // (length rank, start)
  int comp[20], state[21];
  for (int li = lane; li < lens; li += 32) {
    const int len = n - li;
    seg_state(s, len, comp, state);
    for (int i = 0;; ++i) {
      const double p = seg_probability(a, state, len);
      if (p < best) {
        best = p;
        best_at = ((uint64_t)li << 32) | (uint32_t)i;
      }
      if (i + 1 + len > n) break;
      const int out = seg_class(s[i]), in = seg_class(s[i + len]);
      if (out >= 0) {
        state_shrink(state, comp[out]);
        --comp[out];
      }
      if (in >= 0) {
        state_grow(state, comp[in]);
        ++comp[in];
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const uint64_t oa = __shfl_xor_sync(0xffffffffu, best_at, o);
    if (ob < best || (ob == best && oa < best_at)) {
      best = ob;
      best_at = oa;
    }
  }
  int best_left = 0, best_right = n - 1;
  if (best_at != ~0ull) {
    const int len = n - (int)(best_at >> 32);
    best_left = (int)(uint32_t)best_at;
    best_right = len + best_left - 1;
  }
  *left += best_left;
  *right -= n - best_right - 1;
}

struct SegFrame {
  int base, n, i, left_limit;
};

// Masks the low-complexity segments of s[0..n) (n >= the window); every
// lane of the warp runs the same search on the same data (so its branches
// agree), the trimming is split over the lanes, and lane 0 writes the
// masks.  E, when given, holds the entropy of the window starting at every
// position 0 .. n-12 of s (computed before any mask), so the search reads
// H instead of computing it; a frame's H(i) is that of the window starting
// at its position min(i, its length - 12).  Returns false if the search
// nested deeper than the stack.
__device__ bool seg_sequence(const SegArgs &a, uint8_t *s, int n, int lane, const double *E) {
  SegFrame stack[kSegStack];
  int depth = 0;
  stack[0] = {0, n, 0, 0};
  int comp[20], state[21];
  while (depth >= 0) {
    SegFrame f = stack[depth];
    const uint8_t *w = s + f.base;
    bool pushed = false;
    // H over the frame, sliding from position f.i (or read from E)
    auto h_at = [&](int i) {
      return E[f.base + (i < f.n - kSegWindow ? i : f.n - kSegWindow)];
    };
    int start = f.i < f.n - kSegWindow ? f.i : f.n - kSegWindow;
    if (!E) seg_state(w + start, kSegWindow, comp, state);
    for (int i = f.i; i <= f.n - 1; ++i) {
      const int want = i < f.n - kSegWindow ? i : f.n - kSegWindow;
      while (!E && start < want) {  // slide by one
        const int out = seg_class(w[start]), in = seg_class(w[start + kSegWindow]);
        if (out >= 0) {
          state_shrink(state, comp[out]);
          --comp[out];
        }
        if (in >= 0) {
          state_grow(state, comp[in]);
          ++comp[in];
        }
        ++start;
      }
      if ((E ? h_at(i) : seg_entropy(a, state)) > kSegLowCut) continue;
      int lo = i;
      while (lo >= f.left_limit && (E ? h_at(lo) : seg_h(a, w, f.n, lo)) <= kSegHighCut) --lo;
      const int left_i = lo + 1;
      int hi = i;
      while (hi <= f.n - 1 && (E ? h_at(hi) : seg_h(a, w, f.n, hi)) <= kSegHighCut) ++hi;
      const int right_i = hi - 1;
      int left_end = left_i, right_end = right_i;
      seg_trim_warp(a, w + left_end, right_end - left_end + 1, &left_end, &right_end, lane);
      // the mask bit is invisible to seg_class, so the other lanes' reads
      // see the same letters whichever value they load
      if (lane == 0)
        for (int k = left_end; k <= right_end; ++k) s[f.base + k] |= kMaskBit;
      const int next = right_i < right_end ? right_i : right_end;
      const bool child = i < left_end && left_end - left_i >= kSegWindow;
      // the frame resumes after the segment
      stack[depth].i = next + 1;
      stack[depth].left_limit = next + 1;
      if (child) {
        if (depth + 1 >= kSegStack) return false;
        stack[++depth] = {f.base + left_i, left_end - left_i, 0, 0};
        pushed = true;
        break;
      }
      i = next;
      f.left_limit = next + 1;
      // the window restarts at the new position
      start = next + 1 < f.n - kSegWindow ? next + 1 : f.n - kSegWindow;
      if (!E && next + 1 <= f.n - 1) seg_state(w + start, kSegWindow, comp, state);
    }
    if (!pushed) --depth;
  }
  return true;
}

// the sequence of unit u: a frame of a translated query (mode 0) or the
// body of a protein query (mode 1); n = 0 for none
__device__ __forceinline__ uint8_t *unit_of(uint8_t *codes, const uint64_t *offsets,
                                            const uint32_t *lengths, uint64_t u, int mode,
                                            int *n, uint8_t *fallback) {
  if (mode == 0) {
    const uint64_t r = u / 6;
    const int f = (int)(u % 6);
    const uint32_t len = lengths[r];  // bases of the read
    *fallback = kUnknownCode;
    if (len < 3) {
      *n = 0;
      return codes;
    }
    const uint32_t slot = len / 3 + 1;
    *n = (int)((len - (uint32_t)(f % 3)) / 3);
    return codes + offsets[r] + 1 + (uint64_t)f * slot;
  }
  *fallback = 0;
  *n = (int)lengths[u] - 2;
  return codes + offsets[u] + 1;
}

// the letters a caller kept out of the compositions (code + 32) back to
// their codes, masked positions to the unknown code
__device__ __forceinline__ uint8_t finish_code(uint8_t v) {
  return (v & kMaskBit) ? kUnknownCode : ((v & 63) >= 32 ? (uint8_t)((v & 63) - 32) : v);
}

// Pass 1, one thread per sequence: the window entropies only.  A window's
// entropy needs its letter counts in decreasing order, which here come from
// counts-of-counts (how many letters occur v times, v = 12 .. 1) updated in
// O(1) per step, summed in the same order as the sorted counts.  A sequence
// with no window at or below the low cut is finished here (nothing is
// masked); one with such a window gets bit 7 on its first code and is left
// to pass 2.
__global__ void __launch_bounds__(kSegBlock)
    seg_scan_kernel(SegArgs a, uint8_t *__restrict__ codes, const uint64_t *__restrict__ offsets,
                    const uint32_t *__restrict__ lengths, uint64_t units, int mode,
                    uint32_t *__restrict__ status) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < units;
       u += (uint64_t)gridDim.x * blockDim.x) {
    int n;
    uint8_t fallback;
    uint8_t *s = unit_of(codes, offsets, lengths, u, mode, &n, &fallback);
    if (n <= 0) continue;
    if (n < kSegWindow) {
      for (int i = 0; i < n; ++i) s[i] = fallback;
      continue;
    }
    if (n > kSegMaxLength) {
      if (status) atomicAdd(status, 1u);
      for (int i = 0; i < n; ++i) s[i] = finish_code(s[i]);
      continue;
    }
    uint8_t comp[20];
    uint8_t per[kSegWindow + 1];  // per[v]: letters occurring v times
    for (int k = 0; k < 20; ++k) comp[k] = 0;
    for (int v = 0; v <= kSegWindow; ++v) per[v] = 0;
    int total = 0;
    bool marked = false, shifted = false;
    for (int i = 0; i < kSegWindow; ++i) {
      const int k = seg_class(s[i]);
      shifted |= (s[i] & 63) >= 32;
      if (k >= 0) {
        ++comp[k];
        ++total;
      }
    }
    for (int k = 0; k < 20; ++k) ++per[comp[k]];
    for (int start = 0;; ++start) {
      double ent = 0.0;
      if (total == kSegWindow) {
        for (int v = kSegWindow; v >= 1; --v)
          for (int t = 0; t < per[v]; ++t) ent = __dadd_rn(ent, a.entropy12[v]);
      } else if (total > 0) {
        const double r = __ddiv_rn(1.0, (double)total);
        for (int v = total; v >= 1; --v)
          for (int t = 0; t < per[v]; ++t)
            ent = __dadd_rn(ent, __dmul_rn((double)v, a.log_ratio[total][v]));
        ent = __ddiv_rn(__dmul_rn(-ent, r), a.ln2);
      }
      if (ent <= kSegLowCut) {
        marked = true;
        break;
      }
      if (start + kSegWindow >= n) break;
      const int out = seg_class(s[start]), in = seg_class(s[start + kSegWindow]);
      shifted |= (s[start + kSegWindow] & 63) >= 32;
      if (out >= 0) {
        --per[comp[out]];
        --comp[out];
        ++per[comp[out]];
        --total;
      }
      if (in >= 0) {
        --per[comp[in]];
        ++comp[in];
        ++per[comp[in]];
        ++total;
      }
    }
    if (marked) {
      s[0] |= 128;
    } else if (shifted) {
      for (int i = 0; i < n; ++i) s[i] = finish_code(s[i]);
    }
  }
}

// Pass 1 for protein queries (long sequences), one warp per sequence: the
// window starts split into 32 runs, each lane sliding over its own with the
// counts-of-counts of seg_scan_kernel (the same sums in the same order, so
// the same decisions); the sequence is marked when any lane finds a window
// at or below the low cut.
__global__ void __launch_bounds__(kSegBlock)
    seg_scan_warp_kernel(SegArgs a, uint8_t *__restrict__ codes,
                         const uint64_t *__restrict__ offsets,
                         const uint32_t *__restrict__ lengths, uint64_t units, int mode,
                         uint32_t *__restrict__ status) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t u = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; u < units;
       u += warps) {
    int n;
    uint8_t fallback;
    uint8_t *s = unit_of(codes, offsets, lengths, u, mode, &n, &fallback);
    if (n <= 0) continue;
    if (n < kSegWindow) {
      for (int i = lane; i < n; i += 32) s[i] = fallback;
      continue;
    }
    if (n > kSegMaxLength) {
      if (status && lane == 0) atomicAdd(status, 1u);
      for (int i = lane; i < n; i += 32) s[i] = finish_code(s[i]);
      continue;
    }
    bool shifted = false;
    for (int i = lane; i < n; i += 32) shifted |= (s[i] & 63) >= 32;
    const int m = n - kSegWindow + 1;  // window starts 0 .. n-12
    const int run = (m + 31) / 32, p0 = lane * run, p1 = min(p0 + run, m);
    bool low = false;
    if (p0 < p1) {
      uint8_t comp[20];
      uint8_t per[kSegWindow + 1];  // per[v]: letters occurring v times
      for (int k = 0; k < 20; ++k) comp[k] = 0;
      for (int v = 0; v <= kSegWindow; ++v) per[v] = 0;
      int total = 0;
      for (int i = p0; i < p0 + kSegWindow; ++i) {
        const int k = seg_class(s[i]);
        if (k >= 0) {
          ++comp[k];
          ++total;
        }
      }
      for (int k = 0; k < 20; ++k) ++per[comp[k]];
      for (int start = p0;; ++start) {
        double ent = 0.0;
        if (total == kSegWindow) {
          for (int v = kSegWindow; v >= 1; --v)
            for (int t = 0; t < per[v]; ++t) ent = __dadd_rn(ent, a.entropy12[v]);
        } else if (total > 0) {
          const double r = __ddiv_rn(1.0, (double)total);
          for (int v = total; v >= 1; --v)
            for (int t = 0; t < per[v]; ++t)
              ent = __dadd_rn(ent, __dmul_rn((double)v, a.log_ratio[total][v]));
          ent = __ddiv_rn(__dmul_rn(-ent, r), a.ln2);
        }
        if (ent <= kSegLowCut) {
          low = true;
          break;
        }
        if (start + 1 >= p1) break;
        const int out = seg_class(s[start]), in = seg_class(s[start + kSegWindow]);
        if (out >= 0) {
          --per[comp[out]];
          --comp[out];
          ++per[comp[out]];
          --total;
        }
        if (in >= 0) {
          --per[comp[in]];
          ++comp[in];
          ++per[comp[in]];
          ++total;
        }
      }
    }
    const bool marked = __any_sync(0xffffffffu, low);
    shifted = __any_sync(0xffffffffu, shifted);
    if (marked) {
      if (lane == 0) s[0] |= 128;
    } else if (shifted) {
      for (int i = lane; i < n; i += 32) s[i] = finish_code(s[i]);
    }
    __syncwarp();
  }
}

// Pass 2, one warp per sequence pass 1 marked: the whole search
__global__ void __launch_bounds__(kSegBlock)
    seg_search_kernel(SegArgs a, uint8_t *__restrict__ codes, const uint64_t *__restrict__ offsets,
                      const uint32_t *__restrict__ lengths, uint64_t units, int mode,
                      uint32_t *__restrict__ status, int cache) {
  extern __shared__ double ecache[];  // [warps of the block][cache]
  const int lane = threadIdx.x & 31;
  double *E = ecache + (size_t)(threadIdx.x >> 5) * cache;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t u = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; u < units;
       u += warps) {
    int n;
    uint8_t fallback;
    uint8_t *s = unit_of(codes, offsets, lengths, u, mode, &n, &fallback);
    if (n < kSegWindow || n > kSegMaxLength) continue;
    if (!(s[0] & 128)) continue;
    __syncwarp();
    if (lane == 0) s[0] &= 127;
    __syncwarp();
    // the window entropies, lane l sliding over its own run of starts
    const int m = n - kSegWindow + 1;  // window starts 0 .. n-12
    const bool cached = m <= cache;
    if (cached) {
      const int per = (m + 31) / 32, p0 = lane * per, p1 = min(p0 + per, m);
      if (p0 < p1) {
        int comp[20], state[21];
        seg_state(s + p0, kSegWindow, comp, state);
        for (int p = p0;; ++p) {
          E[p] = seg_entropy(a, state);
          if (p + 1 >= p1) break;
          const int out = seg_class(s[p]), in = seg_class(s[p + kSegWindow]);
          if (out >= 0) {
            state_shrink(state, comp[out]);
            --comp[out];
          }
          if (in >= 0) {
            state_grow(state, comp[in]);
            ++comp[in];
          }
        }
      }
      __syncwarp();
    }
    const bool ok = seg_sequence(a, s, n, lane, cached ? E : nullptr);
    __syncwarp();
    if (!ok && lane == 0 && status) atomicAdd(status, 1u);
    for (int i = lane; i < n; i += 32) {
      const uint8_t v = ok ? s[i] : (uint8_t)(s[i] & ~kMaskBit);
      s[i] = finish_code(v);
    }
    __syncwarp();
  }
}

std::once_flag g_tables_once;
SegArgs g_args;
double g_ln_fact_host[kSegMaxLength + 1];
std::mutex g_upload_mutex;
bool g_uploaded[64];

void build_tables() {
  char text[64];
  for (int n = 0; n <= kSegMaxLength; ++n) {
    // ln(n!) from the long-double log-gamma, rounded to 6 decimals through
    // its decimal text (the form of the reference's table)
    snprintf(text, sizeof text, "%.6Lf", n < 2 ? 0.0L : lgammal((long double)n + 1.0L));
    g_ln_fact_host[n] = strtod(text, nullptr);
  }
  g_args.ln2 = std::log(2.0);
  g_args.ln20 = std::log(20.0);
  const double w = kSegWindow;
  g_args.entropy12[0] = 0.0;
  for (int i = 1; i <= kSegWindow; ++i) {
    const double x = i / w;
    g_args.entropy12[i] = -x * std::log(x) / g_args.ln2;
  }
  for (int t = 0; t < kSegWindow; ++t)
    for (int v = 0; v <= kSegWindow; ++v)
      g_args.log_ratio[t][v] = (t > 0 && v > 0 && v <= t) ? std::log(v * (1.0 / (double)t)) : 0.0;
}

int ensure_tables() {
  std::call_once(g_tables_once, build_tables);
  int device = 0;
  GZB_CUDA(cudaGetDevice(&device));
  GZB_CHECK(device >= 0 && device < 64, GZB_ERR_INVALID, "SEG: device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_upload_mutex);
  if (!g_uploaded[device]) {
    GZB_CUDA(cudaMemcpyToSymbol(g_seg_ln_fact, g_ln_fact_host, sizeof(g_ln_fact_host)));
    g_uploaded[device] = true;
  }
  return GZB_OK;
}

int launch_seg(uint8_t *codes, const uint64_t *offsets, const uint32_t *lengths, uint64_t units,
               int mode, uint32_t *status, cudaStream_t stream) {
  GZB_TRY(ensure_tables());
  int device = 0, sms = 148;
  GZB_CUDA(cudaGetDevice(&device));
  GZB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const uint64_t most = (uint64_t)sms * 16;
  if (mode == 0) {  // frames of translated reads: short, one thread each
    const uint64_t want = (units + kSegBlock - 1) / kSegBlock;
    seg_scan_kernel<<<(uint32_t)(want < most ? want : most), kSegBlock, 0, stream>>>(
        g_args, codes, offsets, lengths, units, mode, status);
  } else {  // protein bodies: a warp each
    const uint64_t want = (units + kSegBlock / 32 - 1) / (kSegBlock / 32);
    seg_scan_warp_kernel<<<(uint32_t)(want < most ? want : most), kSegBlock, 0, stream>>>(
        g_args, codes, offsets, lengths, units, mode, status);
  }
  GZB_CUDA(cudaGetLastError());
  const int cache = mode == 0 ? kSegCacheFrames : kSegCacheProteins;
  const int block = mode == 0 ? 128 : 64;
  const uint64_t want2 = (units + block / 32 - 1) / (block / 32);
  const size_t cache_bytes = sizeof(double) * (block / 32) * cache;
  GZB_CUDA(cudaFuncSetAttribute(seg_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)cache_bytes));
  // the warps stride over the sequences, so the grid is what stays resident
  // at once (the caches' shared memory bounds it): one wave, no tail
  int per_sm = 1;
  GZB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, seg_search_kernel, block,
                                                         cache_bytes));
  const uint64_t most2 = (uint64_t)sms * (per_sm > 0 ? per_sm : 1);
  seg_search_kernel<<<(uint32_t)(want2 < most2 ? want2 : most2), block, cache_bytes, stream>>>(
      g_args, codes, offsets, lengths, units, mode, status, cache);
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}

}  // namespace

}  // namespace gzb

extern "C" int gzb_seg_translated_queries(uint8_t *d_queries, const uint64_t *d_query_offsets,
                                          const uint32_t *d_read_lengths,
                                          uint32_t number_queries, uint32_t *d_status,
                                          void *stream) {
  using namespace gzb;
  if (number_queries == 0) return GZB_OK;
  GZB_CHECK(d_queries && d_query_offsets && d_read_lengths, GZB_ERR_INVALID,
            "gzb_seg_translated_queries: null buffer");
  return launch_seg(d_queries, d_query_offsets, d_read_lengths, 6ull * number_queries, 0,
                    d_status, (cudaStream_t)stream);
}

extern "C" int gzb_seg_protein_queries(uint8_t *d_codes, const uint64_t *d_offsets,
                                       const uint32_t *d_lengths, uint32_t number_queries,
                                       uint32_t *d_status, void *stream) {
  using namespace gzb;
  if (number_queries == 0) return GZB_OK;
  GZB_CHECK(d_codes && d_offsets && d_lengths, GZB_ERR_INVALID,
            "gzb_seg_protein_queries: null buffer");
  return launch_seg(d_codes, d_offsets, d_lengths, number_queries, 1, d_status,
                    (cudaStream_t)stream);
}
