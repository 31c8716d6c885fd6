// gzb_operators.cu -- the per-operator C ABI: DistanceCalculatorGpu,
// UngappedExtenderGpu and GappedExtenderGpu of the reference, one handle
// each, with the same host/device split as the reference methods.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <new>

#include "ghostz_b200.h"
#include "gzb_common.h"
#include "gzb_kernels.cuh"

namespace gzb {

static thread_local char g_last_error[512] = "";

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

// --------------------------------------------------------------------------
// kernels

// Windows of up to kWordWindow bytes are fetched as the naturally aligned
// 32-bit words that hold them: at most four words, and only the words that
// hold at least one byte of the window (so no load reaches past the pages
// the window lies in).  w[] receives the window's bytes from byte 0 of w[0].
constexpr int kWordWindow = 13;

__device__ __forceinline__ void window_words(const uint8_t *p, int L, uint32_t w[4]) {
  const uintptr_t a = (uintptr_t)p;
  const uint32_t *base = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
  const int off = (int)(a & 3);
  const int nw = (off + L + 3) >> 2;
  uint32_t r[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) r[j] = j < nw ? __ldg(base + j) : 0u;
  const unsigned sh = 8u * (unsigned)off;
  w[0] = __funnelshift_r(r[0], r[1], sh);
  w[1] = __funnelshift_r(r[1], r[2], sh);
  w[2] = __funnelshift_r(r[2], r[3], sh);
  w[3] = __funnelshift_r(r[3], 0u, sh);
}

// Reduced-alphabet mismatches of two windows held as words (L <= kWordWindow).
__device__ __forceinline__ int word_distance(const uint32_t *a, const uint32_t *b, int L,
                                             const uint8_t *map) {
  int m = 0;
#pragma unroll
  for (int i = 0; i < kWordWindow; ++i)
    if (i < L)
      m += map[(a[i >> 2] >> (8 * (i & 3))) & 0xFF] != map[(b[i >> 2] >> (8 * (i & 3))) & 0xFF];
  return m;
}

// Distance of every seed: the reduced-alphabet mismatches over the L window
// centred on the seed's query and database positions.  A thread takes two
// seeds a pass (their loads in flight together); windows up to kWordWindow
// bytes are read as words, longer ones byte by byte.
__global__ void distance_kernel(const uint8_t *__restrict__ q,
                                const uint8_t *__restrict__ d,
                                const uint8_t *__restrict__ map_g, int L,
                                size_t n, const uint32_t *__restrict__ qc,
                                const uint32_t *__restrict__ dc,
                                int8_t *__restrict__ out) {
  __shared__ uint8_t map[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) map[i] = i < 32 ? map_g[i] : 0;
  __syncthreads();
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const int half = L / 2;
  if (L > kWordWindow) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride)
      out[i] = (int8_t)window_distance(q + qc[i], d + dc[i], L, map);
    return;
  }
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += 2 * stride) {
    const size_t j = i + stride;
    const bool two = j < n;
    const uint32_t qa = qc[i], da = dc[i];
    const uint32_t qb = two ? qc[j] : qa, db = two ? dc[j] : da;
    uint32_t wqa[4], wda[4], wqb[4], wdb[4];
    window_words(q + qa - half, L, wqa);
    window_words(d + da - half, L, wda);
    window_words(q + qb - half, L, wqb);
    window_words(d + db - half, L, wdb);
    out[i] = (int8_t)word_distance(wqa, wda, L, map);
    if (two) out[j] = (int8_t)word_distance(wqb, wdb, L, map);
  }
}

// Ungapped extension with trigger, one thread per seed.
__global__ void ungapped_trigger_kernel(
    const uint8_t *__restrict__ q, const uint8_t *__restrict__ d, int delim,
    const int32_t *__restrict__ matrix, int number_letters, int stride,
    const int32_t *__restrict__ cutoffs, const int32_t *__restrict__ triggers,
    size_t n, const uint32_t *__restrict__ qid,
    const uint32_t *__restrict__ qpos, const uint32_t *__restrict__ dpos,
    int8_t *__restrict__ flags) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t id = qid[i];
    int steps = 0;
    flags[i] = ungapped_hit(q + qpos[i], d + dpos[i], delim, sm, cutoffs[id],
                            triggers[id], &steps)
                   ? 1
                   : 0;
  }
}

// set[start[i]] = i (the run-start scatter of SetQuerySeeds).
__global__ void scatter_starts_kernel(size_t nseeds, const uint32_t *starts,
                                      size_t size, uint32_t *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nseeds;
       i += (size_t)gridDim.x * blockDim.x)
    if (starts[i] < size) out[starts[i]] = (uint32_t)i;
}

// In-place inclusive max-scan of one block-sized tile; tile maxima are
// written to `tile_max`.  Hand-written replacement of the CUB max-scan.
template <int B>
__global__ void max_scan_tiles(uint32_t *a, size_t n, uint32_t *tile_max) {
  __shared__ uint32_t warp_max[B / 32];
  const size_t i = blockIdx.x * (size_t)B + threadIdx.x;
  uint32_t v = i < n ? a[i] : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = max(v, t);
  }
  if (lane == 31) warp_max[w] = v;
  __syncthreads();
  if (w == 0) {
    uint32_t x = lane < B / 32 ? warp_max[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x = max(x, t);
    }
    if (lane < B / 32) warp_max[lane] = x;
  }
  __syncthreads();
  if (w > 0) v = max(v, warp_max[w - 1]);
  if (i < n) a[i] = v;
  if (threadIdx.x == B - 1 && tile_max) tile_max[blockIdx.x] = v;
}

template <int B>
__global__ void max_scan_apply(uint32_t *a, size_t n, const uint32_t *tile_prefix) {
  const size_t i = blockIdx.x * (size_t)B + threadIdx.x;
  if (blockIdx.x > 0 && i < n) a[i] = max(a[i], tile_prefix[blockIdx.x - 1]);
}

// Per-seed query id / concatenated position through the query-seed id.
__global__ void set_query_seeds_kernel(size_t size, const uint32_t *list_qid,
                                       const uint32_t *list_qpos,
                                       const uint32_t *seed_ids,
                                       const uint32_t *run_of,
                                       uint32_t *out_qid, uint32_t *out_qpos) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < size;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t s = seed_ids[run_of[i]];
    out_qid[i] = list_qid[s];
    out_qpos[i] = list_qpos[s];
  }
}

__global__ void gather_kernel(size_t n, const uint32_t *idx, const uint32_t *src,
                              uint32_t *dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

// Gapped extension kernels.  Every extension first runs on one thread
// (gapped_lane_kernel); the few whose band outgrows the thread's shared
// buffer go to one warp each (gapped_warp_kernel), and any left after that to
// the serial kernel with a band in global memory.  Extension lists live in
// device memory with device-side counts, so the three launches need no host
// synchronisation.
constexpr int kLaneBlock = 128;
static_assert(kLaneBlock == 128, "the lane band's residue layout assumes four warps per block");
constexpr int kBandW = 256;
constexpr int kSerialThreads = 4 * 128;
constexpr int kSerialBand = 1 << 15;  // columns per fallback thread
constexpr int kGappedWarps = 8;

__device__ __forceinline__ void store_result(uint32_t e, uint32_t q, uint32_t d,
                                             const GappedOut &o, uint32_t *qpos,
                                             uint32_t *dpos, int32_t *scores) {
  qpos[e] = q + (uint32_t)o.pos0;
  dpos[e] = d + (uint32_t)o.pos1;
  scores[e] = o.score;
}

__global__ void __launch_bounds__(kLaneBlock)
gapped_lane_kernel(GappedJob job, const int32_t *__restrict__ matrix, int number_letters,
                   int stride, size_t n, const uint32_t *__restrict__ order, int reverse,
                   const uint8_t *__restrict__ dir, uint32_t *qpos, uint32_t *dpos,
                   int32_t *scores, uint32_t *spill, uint32_t *spill_count,
                   unsigned long long *cells_total, uint32_t *cells_out, const uint64_t *n_dev) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  __shared__ uint32_t cells_s[kLaneW * kLaneBlock];
  __shared__ uint8_t res_s[kLaneW * kLaneBlock];
  if (n_dev) n = *n_dev;
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  LaneBand<kLaneW> band(cells_s, res_s, kLaneBlock, (int)threadIdx.x);
  unsigned long long cells = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t e = order ? order[i] : (uint32_t)i;
    const bool rev = dir ? dir[e] != 0 : reverse != 0;
    const uint32_t q = qpos[e], d = dpos[e];
    GappedOut o = gapped_extend_lane(job, sm, band, q, d, rev);
    if (o.overflow) {
      spill[atomicAdd(spill_count, 1u)] = e;
      if (cells_out) cells_out[e] = 0xFFFFFFFFu;
    } else {
      cells += o.cells;
      store_result(e, q, d, o, qpos, dpos, scores);
      if (cells_out) cells_out[e] = (uint32_t)o.cells;
    }
  }
  cells += __shfl_down_sync(0xffffffffu, cells, 16);
  cells += __shfl_down_sync(0xffffffffu, cells, 8);
  cells += __shfl_down_sync(0xffffffffu, cells, 4);
  cells += __shfl_down_sync(0xffffffffu, cells, 2);
  cells += __shfl_down_sync(0xffffffffu, cells, 1);
  if ((threadIdx.x & 31) == 0 && cells) atomicAdd(cells_total, cells);
}

// Flattened one-thread-per-extension kernel over a device work queue
// (persistent blocks; `order` optional).  Dynamic shared memory:
// kFlatW * blockDim.x int2.
__global__ void __launch_bounds__(kFlatBlock)
gapped_flat_kernel(GappedJob job, const int32_t *__restrict__ matrix, int number_letters,
                   int stride, uint64_t n, const uint32_t *__restrict__ order,
                   unsigned long long *queue, int reverse, const uint8_t *__restrict__ dir,
                   uint32_t *qpos, uint32_t *dpos, int32_t *scores, uint32_t *spill,
                   uint32_t *spill_count, unsigned long long *cells_total,
                   uint32_t *cells_out, int book_threshold, const uint64_t *n_dev) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  extern __shared__ int2 flat_band[];
  if (n_dev) n = *n_dev;
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  FlatOut o{qpos, dpos, scores, spill, spill_count, cells_out};
  const unsigned long long c = gapped_flat(job, sm, flat_band + threadIdx.x, (int)blockDim.x, n,
                                           order, queue, reverse, dir, o, book_threshold);
  if (c) atomicAdd(cells_total, c);
}

// Nested one-thread-per-extension kernel over a device work queue:
// persistent blocks; each warp takes the next 32 extensions of `order` (or
// of extension order) and runs them to completion together, so extensions
// of similar cost placed next to each other keep the warp's lanes busy.
// cells_out (optional) records every extension's DP cells, UINT32_MAX when
// it was handed to the fallback.
__global__ void __launch_bounds__(kLaneBlock)
gapped_lane_queue_kernel(GappedJob job, const int32_t *__restrict__ matrix, int number_letters,
                         int stride, uint64_t n, const uint32_t *__restrict__ order,
                         unsigned long long *queue, int reverse, const uint8_t *__restrict__ dir,
                         uint32_t *qpos, uint32_t *dpos, int32_t *scores, uint32_t *spill,
                         uint32_t *spill_count, unsigned long long *cells_total,
                         uint32_t *cells_out, const uint64_t *n_dev) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  __shared__ uint32_t cells_s[kLaneW * kLaneBlock];
  __shared__ uint8_t res_s[kLaneW * kLaneBlock];
  if (n_dev) n = *n_dev;
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  LaneBand<kLaneW> band(cells_s, res_s, kLaneBlock, (int)threadIdx.x);
  const int lane = threadIdx.x & 31;
  unsigned long long cells = 0;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(queue, 32ull);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const uint64_t i = base + lane;
    if (i < n) {
      const uint32_t e = order ? order[i] : (uint32_t)i;
      const bool rev = dir ? dir[e] != 0 : reverse != 0;
      const uint32_t q = qpos[e], d = dpos[e];
      GappedOut o = gapped_extend_lane(job, sm, band, q, d, rev);
      if (o.overflow) {
        spill[atomicAdd(spill_count, 1u)] = e;
        if (cells_out) cells_out[e] = 0xFFFFFFFFu;
      } else {
        cells += o.cells;
        store_result(e, q, d, o, qpos, dpos, scores);
        if (cells_out) cells_out[e] = o.cells > 0xFFFFFFFEull ? 0xFFFFFFFEu : (uint32_t)o.cells;
      }
    }
    __syncwarp();
  }
  cells += __shfl_down_sync(0xffffffffu, cells, 16);
  cells += __shfl_down_sync(0xffffffffu, cells, 8);
  cells += __shfl_down_sync(0xffffffffu, cells, 4);
  cells += __shfl_down_sync(0xffffffffu, cells, 2);
  cells += __shfl_down_sync(0xffffffffu, cells, 1);
  if (lane == 0 && cells) atomicAdd(cells_total, cells);
}

// Row-granular work queue: every lane runs its own extension one database
// row per step and takes the next extension from the queue once its own has
// ended, so the lanes of a warp wait for each other only within a row (the
// widest band of the step), never for the longest extension.  A lane whose
// extension ended writes it out at once and then idles until
// `refill_threshold` lanes of its warp are idle (or no lane has work left):
// those lanes then fetch, load and start their next extensions together, so
// one round of memory latency and one pass of the set-up code serve them all.
// W: band columns per lane (the GZB_TILE_BAND_WIDTH tile): a narrower band
// fits more blocks on an SM and hands more extensions to the warp kernel.
// Bands up to 64 columns live in static shared memory (the fastest form
// measured); wider ones, above the 48 KB static limit, in dynamic shared
// memory, rows_band_bytes(W) per block.
__host__ __device__ constexpr bool rows_band_static(int W) { return W <= 64; }
constexpr size_t rows_band_bytes(int W) {
  return rows_band_static(W) ? 0 : (size_t)W * kLaneBlock * 5;
}

template <int W>
__global__ void __launch_bounds__(kLaneBlock)
gapped_rows_kernel(GappedJob job, const int32_t *__restrict__ matrix, int number_letters,
                   int stride, uint64_t n, const uint32_t *__restrict__ order,
                   unsigned long long *queue, int reverse, const uint8_t *__restrict__ dir,
                   uint32_t *qpos, uint32_t *dpos, int32_t *scores, uint32_t *spill,
                   uint32_t *spill_count, unsigned long long *cells_total,
                   uint32_t *cells_out, int refill_threshold, const uint64_t *n_dev) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  constexpr bool kStatic = rows_band_static(W);
  __shared__ uint32_t cells_st[kStatic ? W * kLaneBlock : 1];
  __shared__ uint8_t res_st[kStatic ? W * kLaneBlock : 1];
  extern __shared__ __align__(16) uint8_t rows_band[];
  // [W][kLaneBlock] each
  uint32_t *cells_s = kStatic ? cells_st : reinterpret_cast<uint32_t *>(rows_band);
  uint8_t *res_s = kStatic ? res_st : rows_band + (size_t)W * kLaneBlock * 4;
  if (n_dev) n = *n_dev;
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  LaneBand<W> band(cells_s, res_s, kLaneBlock, (int)threadIdx.x);
  LaneExt x;
  uint32_t e = 0, q = 0, d = 0;
  bool have = false, done = false;
  unsigned long long cells = 0;
  for (;;) {
    int st = kLaneRunning;
    if (have) st = lane_row(job, sm, band, x);
    const unsigned idle = __ballot_sync(0xffffffffu, !done && (!have || st != kLaneRunning));
    const unsigned busy = __ballot_sync(0xffffffffu, have && st == kLaneRunning);
    if (idle == 0 && busy == 0) break;
    const bool refill = __popc(idle) >= refill_threshold || busy == 0;
    while (have ? st != kLaneRunning : (refill && !done)) {
      if (have) {  // the extension ended: write it out
        if (st == kLaneOverflow || x.ovf) {
          spill[atomicAdd(spill_count, 1u)] = e;
          if (cells_out) cells_out[e] = 0xFFFFFFFFu;
        } else {
          cells += x.cells;
          qpos[e] = q + (uint32_t)x.mp0;
          dpos[e] = d + (uint32_t)x.mp1;
          scores[e] = x.maxs;
          if (cells_out) cells_out[e] = x.cells;
        }
        have = false;
        st = kLaneRunning;
        if (!refill) break;
      }
      if (!flat_fetch(queue, n, order, &e)) {
        done = true;
        break;
      }
      const bool rev = dir ? dir[e] != 0 : reverse != 0;
      q = qpos[e];
      d = dpos[e];
      st = lane_init(job, band, x, job.query + q, job.db + d, rev);
      have = true;
    }
  }
  cells += __shfl_down_sync(0xffffffffu, cells, 16);
  cells += __shfl_down_sync(0xffffffffu, cells, 8);
  cells += __shfl_down_sync(0xffffffffu, cells, 4);
  cells += __shfl_down_sync(0xffffffffu, cells, 2);
  cells += __shfl_down_sync(0xffffffffu, cells, 1);
  if ((threadIdx.x & 31) == 0 && cells) atomicAdd(cells_total, cells);
}

// Row-step refill with extensions dealt round-robin: lane t of the grid
// runs extensions order[t], order[t + T], order[t + 2T], ... (T threads),
// one database row per step like gapped_rows_kernel, and loads the
// positions of its next extension while the current one runs.
__global__ void __launch_bounds__(kLaneBlock)
gapped_deal_kernel(GappedJob job, const int32_t *__restrict__ matrix, int number_letters,
                   int stride, uint64_t n, const uint32_t *__restrict__ order, int reverse,
                   const uint8_t *__restrict__ dir, uint32_t *qpos, uint32_t *dpos,
                   int32_t *scores, uint32_t *spill, uint32_t *spill_count,
                   unsigned long long *cells_total, uint32_t *cells_out, const uint64_t *n_dev) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  __shared__ uint32_t cells_s[kLaneW * kLaneBlock];
  __shared__ uint8_t res_s[kLaneW * kLaneBlock];
  if (n_dev) n = *n_dev;
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  LaneBand<kLaneW> band(cells_s, res_s, kLaneBlock, (int)threadIdx.x);
  const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  // the next extension of this lane, loaded one extension ahead
  uint32_t ne = 0, nq = 0, nd = 0;
  bool nrev = false;
  auto load_next = [&](uint64_t k) {
    if (k < n) {
      ne = order ? order[k] : (uint32_t)k;
      nq = qpos[ne];
      nd = dpos[ne];
      nrev = dir ? dir[ne] != 0 : reverse != 0;
    }
  };
  load_next(i);
  LaneExt x;
  uint32_t e = 0, q = 0, d = 0;
  bool have = false;
  unsigned long long cells = 0;
  for (;;) {
    int st = kLaneRunning;
    if (have) st = lane_row(job, sm, band, x);
    while (st != kLaneRunning || (!have && i < n)) {
      if (have) {  // the extension ended: write it out
        if (st == kLaneOverflow || x.ovf) {
          spill[atomicAdd(spill_count, 1u)] = e;
          if (cells_out) cells_out[e] = 0xFFFFFFFFu;
        } else {
          cells += x.cells;
          qpos[e] = q + (uint32_t)x.mp0;
          dpos[e] = d + (uint32_t)x.mp1;
          scores[e] = x.maxs;
          if (cells_out) cells_out[e] = x.cells;
        }
        have = false;
        i += T;
      }
      if (i >= n) break;
      e = ne;
      q = nq;
      d = nd;
      const bool rev = nrev;
      load_next(i + T);
      st = lane_init(job, band, x, job.query + q, job.db + d, rev);
      have = true;
    }
    if (!__any_sync(0xffffffffu, have)) break;
  }
  cells += __shfl_down_sync(0xffffffffu, cells, 16);
  cells += __shfl_down_sync(0xffffffffu, cells, 8);
  cells += __shfl_down_sync(0xffffffffu, cells, 4);
  cells += __shfl_down_sync(0xffffffffu, cells, 2);
  cells += __shfl_down_sync(0xffffffffu, cells, 1);
  if ((threadIdx.x & 31) == 0 && cells) atomicAdd(cells_total, cells);
}

// process-wide tile defaults (gzb_set_tile_parameter)
GappedTile g_tile = {GZB_GAPPED_KERNEL_ROWS, 4, GZB_ORDER_MODEL, GZB_SEED_WALKER_UNIT, kLaneW};

template <typename K>
static int persistent_blocks(K kernel, int block, size_t smem, uint64_t n, uint64_t *blocks) {
  int dev = 0, sms = 148, per_sm = 1;
  GZB_CUDA(cudaGetDevice(&dev));
  GZB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GZB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem));
  if (per_sm < 1) per_sm = 1;
  uint64_t b = (uint64_t)sms * per_sm;
  const uint64_t need = (n + block - 1) / block;
  if (need < b) b = need ? need : 1;
  *blocks = b;
  return GZB_OK;
}

// G lanes per extension (gapped_extend_group), each group pulling the next
// extension from the work queue as soon as its own ends; a band wider than
// kGroupBandW columns goes to the spill list (then the warp kernel).
constexpr int kGroupBlock = 128;
constexpr int kGroupBandW = 64;

template <int G>
__global__ void __launch_bounds__(kGroupBlock)
gapped_group_kernel(GappedJob job, const int32_t *__restrict__ matrix, int number_letters,
                    int stride, uint64_t n, const uint32_t *__restrict__ order,
                    unsigned long long *queue, int reverse, const uint8_t *__restrict__ dir,
                    uint32_t *qpos, uint32_t *dpos, int32_t *scores, uint32_t *spill,
                    uint32_t *spill_count, unsigned long long *cells_total, uint32_t *cells_out,
                    const uint64_t *n_dev) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  __shared__ int2 bands[kGroupBlock / G][kGroupBandW];
  if (n_dev) n = *n_dev;
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  const LaneGroup<G> g;
  const int grp = threadIdx.x / G;
  unsigned long long cells = 0;
  for (;;) {
    uint32_t e = 0;
    int got = 0;
    if (g.lane == 0) got = flat_fetch(queue, n, order, &e) ? 1 : 0;
    got = g.at(got, 0);
    if (!got) break;
    e = (uint32_t)g.at((int)e, 0);
    const bool rev = dir ? dir[e] != 0 : reverse != 0;
    const uint32_t q = qpos[e], d = dpos[e];
    const GappedOut o = gapped_extend_group<G, kGroupBandW>(job, sm, bands[grp], q, d, rev);
    if (g.lane == 0) {
      if (o.overflow) {
        spill[atomicAdd(spill_count, 1u)] = e;
        if (cells_out) cells_out[e] = 0xFFFFFFFFu;
      } else {
        cells += o.cells;
        store_result(e, q, d, o, qpos, dpos, scores);
        if (cells_out) cells_out[e] = (uint32_t)o.cells;
      }
    }
    g.sync();
  }
  cells += __shfl_down_sync(0xffffffffu, cells, 16);
  cells += __shfl_down_sync(0xffffffffu, cells, 8);
  cells += __shfl_down_sync(0xffffffffu, cells, 4);
  cells += __shfl_down_sync(0xffffffffu, cells, 2);
  cells += __shfl_down_sync(0xffffffffu, cells, 1);
  if ((threadIdx.x & 31) == 0 && cells) atomicAdd(cells_total, cells);
}

template <int G>
static int launch_gapped_group(const GappedJob &job, const int32_t *matrix, int number_letters,
                               int stride, uint64_t n, const uint32_t *order,
                               unsigned long long *queue, int reverse, const uint8_t *dir,
                               uint32_t *qpos, uint32_t *dpos, int32_t *scores, uint32_t *spill,
                               uint32_t *spill_count, unsigned long long *cells_total,
                               uint32_t *cells_out, cudaStream_t s, const uint64_t *n_dev) {
  uint64_t blocks = 1;
  GZB_TRY(persistent_blocks(gapped_group_kernel<G>, kGroupBlock, 0, n * G, &blocks));
  gapped_group_kernel<G><<<(unsigned)blocks, kGroupBlock, 0, s>>>(
      job, matrix, number_letters, stride, n, order, queue, reverse, dir, qpos, dpos, scores,
      spill, spill_count, cells_total, cells_out, n_dev);
  return GZB_OK;
}

template <int W>
static int launch_gapped_rows(const GappedTile &tile, const GappedJob &job, const int32_t *matrix,
                              int number_letters, int stride, uint64_t n, const uint32_t *order,
                              unsigned long long *queue, int reverse, const uint8_t *dir,
                              uint32_t *qpos, uint32_t *dpos, int32_t *scores, uint32_t *spill,
                              uint32_t *spill_count, unsigned long long *cells_total,
                              uint32_t *cells_out, cudaStream_t s, const uint64_t *n_dev) {
  const size_t smem = rows_band_bytes(W);
  if (smem)
    GZB_CUDA(cudaFuncSetAttribute(gapped_rows_kernel<W>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  uint64_t blocks = 1;
  GZB_TRY(persistent_blocks(gapped_rows_kernel<W>, kLaneBlock, smem, n, &blocks));
  gapped_rows_kernel<W><<<(unsigned)blocks, kLaneBlock, smem, s>>>(
      job, matrix, number_letters, stride, n, order, queue, reverse, dir, qpos, dpos, scores,
      spill, spill_count, cells_total, cells_out, tile.book_threshold, n_dev);
  return GZB_OK;
}

int launch_gapped_thread(const GappedTile &tile, const GappedJob &job, const int32_t *matrix,
                         int number_letters, int stride, uint64_t n, const uint32_t *order,
                         unsigned long long *queue, int reverse, const uint8_t *dir,
                         uint32_t *qpos, uint32_t *dpos, int32_t *scores, uint32_t *spill,
                         uint32_t *spill_count, unsigned long long *cells_total,
                         uint32_t *cells_out, cudaStream_t s, const uint64_t *n_dev) {
  // with n_dev the count is read on the device and n is its upper bound
  // (grids sized for n)
  GZB_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s));
  uint64_t blocks = 1;
  const bool group = tile.kernel >= GZB_GAPPED_KERNEL_GROUP4 &&
                     tile.kernel <= GZB_GAPPED_KERNEL_GROUP32 && warp_path_exact(job.cutoff);
  if (group) {
    const int G = 4 << (tile.kernel - GZB_GAPPED_KERNEL_GROUP4);
    if (G == 4)
      GZB_TRY(launch_gapped_group<4>(job, matrix, number_letters, stride, n, order, queue,
                                     reverse, dir, qpos, dpos, scores, spill, spill_count,
                                     cells_total, cells_out, s, n_dev));
    else if (G == 8)
      GZB_TRY(launch_gapped_group<8>(job, matrix, number_letters, stride, n, order, queue,
                                     reverse, dir, qpos, dpos, scores, spill, spill_count,
                                     cells_total, cells_out, s, n_dev));
    else if (G == 16)
      GZB_TRY(launch_gapped_group<16>(job, matrix, number_letters, stride, n, order, queue,
                                      reverse, dir, qpos, dpos, scores, spill, spill_count,
                                      cells_total, cells_out, s, n_dev));
    else
      GZB_TRY(launch_gapped_group<32>(job, matrix, number_letters, stride, n, order, queue,
                                      reverse, dir, qpos, dpos, scores, spill, spill_count,
                                      cells_total, cells_out, s, n_dev));
  } else if (tile.kernel == GZB_GAPPED_KERNEL_DEAL) {
    GZB_TRY(persistent_blocks(gapped_deal_kernel, kLaneBlock, 0, n, &blocks));
    gapped_deal_kernel<<<(unsigned)blocks, kLaneBlock, 0, s>>>(
        job, matrix, number_letters, stride, n, order, reverse, dir, qpos, dpos, scores, spill,
        spill_count, cells_total, cells_out, n_dev);
  } else if (tile.kernel == GZB_GAPPED_KERNEL_STATIC) {
    // one launch, extensions dealt to threads round-robin, no work queue
    blocks = (n + kLaneBlock - 1) / kLaneBlock;
    if (blocks > 148 * 40) blocks = 148 * 40;
    gapped_lane_kernel<<<(unsigned)blocks, kLaneBlock, 0, s>>>(
        job, matrix, number_letters, stride, n, order, reverse, dir, qpos, dpos, scores, spill,
        spill_count, cells_total, cells_out, n_dev);
  } else if (tile.kernel == GZB_GAPPED_KERNEL_ROWS || tile.kernel >= GZB_GAPPED_KERNEL_GROUP4) {
    // (a group kernel's X-drop outside the warp DP's exact range runs here)
    if (tile.band_width == 32)
      GZB_TRY(launch_gapped_rows<32>(tile, job, matrix, number_letters, stride, n, order, queue,
                                     reverse, dir, qpos, dpos, scores, spill, spill_count,
                                     cells_total, cells_out, s, n_dev));
    else if (tile.band_width == 128)
      GZB_TRY(launch_gapped_rows<128>(tile, job, matrix, number_letters, stride, n, order,
                                      queue, reverse, dir, qpos, dpos, scores, spill,
                                      spill_count, cells_total, cells_out, s, n_dev));
    else
      GZB_TRY(launch_gapped_rows<64>(tile, job, matrix, number_letters, stride, n, order, queue,
                                     reverse, dir, qpos, dpos, scores, spill, spill_count,
                                     cells_total, cells_out, s, n_dev));
  } else if (tile.kernel == GZB_GAPPED_KERNEL_LANE) {
    GZB_TRY(persistent_blocks(gapped_lane_queue_kernel, kLaneBlock, 0, n, &blocks));
    gapped_lane_queue_kernel<<<(unsigned)blocks, kLaneBlock, 0, s>>>(
        job, matrix, number_letters, stride, n, order, queue, reverse, dir, qpos, dpos, scores,
        spill, spill_count, cells_total, cells_out, n_dev);
  } else if (tile.kernel == GZB_GAPPED_KERNEL_FLAT) {
    const size_t smem = sizeof(int2) * (size_t)kFlatW * kFlatBlock;
    GZB_CUDA(cudaFuncSetAttribute(gapped_flat_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    GZB_TRY(persistent_blocks(gapped_flat_kernel, kFlatBlock, smem, n, &blocks));
    gapped_flat_kernel<<<(unsigned)blocks, kFlatBlock, smem, s>>>(
        job, matrix, number_letters, stride, n, order, queue, reverse, dir, qpos, dpos, scores,
        spill, spill_count, cells_total, cells_out, tile.book_threshold, n_dev);
  }
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}

// One warp per listed extension (shared circular band of kBandW columns).
__global__ void __launch_bounds__(kGappedWarps * 32)
gapped_warp_kernel(GappedJob job, const int32_t *__restrict__ matrix, int number_letters,
                   int stride, const uint32_t *list, const uint32_t *list_count,
                   int reverse, const uint8_t *__restrict__ dir, uint32_t *qpos,
                   uint32_t *dpos, int32_t *scores, uint32_t *spill, uint32_t *spill_count,
                   unsigned long long *cells_total) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  __shared__ int2 bands[kGappedWarps][kBandW];
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t n = *list_count;
  unsigned long long cells = 0;
  for (size_t i = blockIdx.x * (size_t)kGappedWarps + w; i < n;
       i += (size_t)gridDim.x * kGappedWarps) {
    const uint32_t e = list[i];
    const bool rev = dir ? dir[e] != 0 : reverse != 0;
    const uint32_t q = qpos[e], d = dpos[e];
    GappedOut o = gapped_extend_warp<kBandW>(job, sm, bands[w], kBandW - 1, q, d, rev);
    if (o.overflow) {
      if (lane == 0) spill[atomicAdd(spill_count, 1u)] = e;
    } else {
      cells += o.cells;
      if (lane == 0) store_result(e, q, d, o, qpos, dpos, scores);
    }
    __syncwarp();
  }
  if (lane == 0 && cells) atomicAdd(cells_total, cells);
}

// Serial fallback over a listed set, one thread each, with a global
// circular band of (wmask+1) columns per thread.
__global__ void gapped_serial_kernel(GappedJob job, const int32_t *__restrict__ matrix,
                                     int number_letters, int stride, const uint32_t *list,
                                     const uint32_t *list_count, int reverse,
                                     const uint8_t *__restrict__ dir, uint32_t *qpos,
                                     uint32_t *dpos, int32_t *scores, int2 *band_pool,
                                     int wmask, unsigned long long *cells_total,
                                     uint32_t *too_long_count) {
  __shared__ int sm[kMatrixStride * kMatrixStride];
  load_matrix(sm, matrix, number_letters, stride);
  __syncthreads();
  const size_t count = *list_count;
  const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  int2 *band = band_pool + tid * (size_t)(wmask + 1);
  unsigned long long cells = 0;
  for (size_t i = tid; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t e = list[i];
    const bool rev = dir ? dir[e] != 0 : reverse != 0;
    const uint32_t q = qpos[e], d = dpos[e];
    bool too_long = false;
    GappedOut o = gapped_extend_serial(job, sm, band, wmask, q, d, rev, &too_long);
    if (too_long) {
      atomicAdd(too_long_count, 1u);
      continue;
    }
    cells += o.cells;
    store_result(e, q, d, o, qpos, dpos, scores);
  }
  if (cells) atomicAdd(cells_total, cells);
}

static unsigned grid_for(size_t n, int block, int max_blocks = 148 * 16) {
  size_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > (size_t)max_blocks) g = max_blocks;
  return (unsigned)g;
}

}  // namespace gzb

using namespace gzb;

// --------------------------------------------------------------------------
// C ABI: errors

extern "C" const char *gzb_error_string(int code) {
  switch (code) {
    case GZB_OK: return "ok";
    case GZB_ERR_INVALID: return "invalid argument or state";
    case GZB_ERR_CUDA: return "CUDA runtime error";
    case GZB_ERR_NOMEM: return "out of memory";
    case GZB_ERR_OVERFLOW: return "size exceeds a limit";
    case GZB_ERR_TIMEOUT: return "bounded device wait ran out";
    default: return "unknown error";
  }
}

extern "C" const char *gzb_last_error(void) { return g_last_error; }
extern "C" int gzb_version(void) { return 10000; }

// --------------------------------------------------------------------------
// DistanceCalculatorGpu

struct gzb_distance_calculator {
  const uint8_t *queries = nullptr;
  const uint8_t *db = nullptr;
  const uint8_t *map = nullptr;
  uint32_t L = 0;
};

extern "C" int gzb_distance_calculator_create(gzb_distance_calculator **out) {
  GZB_CHECK(out, GZB_ERR_INVALID, "null output handle");
  *out = new (std::nothrow) gzb_distance_calculator();
  GZB_CHECK(*out, GZB_ERR_NOMEM, "host allocation failed");
  return GZB_OK;
}
extern "C" int gzb_distance_calculator_destroy(gzb_distance_calculator *h) {
  delete h;
  return GZB_OK;
}
extern "C" int gzb_distance_calculator_set_queries(gzb_distance_calculator *h,
                                                   const uint8_t *d) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->queries = d;
  return GZB_OK;
}
extern "C" int gzb_distance_calculator_set_database(gzb_distance_calculator *h,
                                                    const uint8_t *d) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->db = d;
  return GZB_OK;
}
extern "C" int gzb_distance_calculator_set_reduced_code_map(
    gzb_distance_calculator *h, const uint8_t *d) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->map = d;
  return GZB_OK;
}
extern "C" int gzb_distance_calculator_set_subsequence_length(
    gzb_distance_calculator *h, uint32_t L) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->L = L;
  return GZB_OK;
}
extern "C" int gzb_distance_calculator_calculate_distances_async(
    gzb_distance_calculator *h, size_t size, const uint32_t *qc,
    const uint32_t *dc, int8_t *out, uint32_t *d_qc, uint32_t *d_dc,
    int8_t *d_out, void *stream) {
  GZB_CHECK(h && h->queries && h->db && h->map, GZB_ERR_INVALID,
            "distance calculator not set up");
  GZB_CHECK(h->L > 0 && h->L <= 64, GZB_ERR_INVALID, "bad subsequence length %u", h->L);
  if (size == 0) return GZB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (qc) GZB_CUDA(cudaMemcpyAsync(d_qc, qc, 4 * size, cudaMemcpyDefault, s));
  if (dc) GZB_CUDA(cudaMemcpyAsync(d_dc, dc, 4 * size, cudaMemcpyDefault, s));
  distance_kernel<<<grid_for(size, 256), 256, 0, s>>>(h->queries, h->db, h->map,
                                                     (int)h->L, size, d_qc, d_dc, d_out);
  GZB_CUDA(cudaGetLastError());
  if (out) GZB_CUDA(cudaMemcpyAsync(out, d_out, size, cudaMemcpyDefault, s));
  return GZB_OK;
}

// --------------------------------------------------------------------------
// UngappedExtenderGpu

struct gzb_ungapped_extender {
  const uint32_t *list_qid = nullptr, *list_qpos = nullptr;
  uint8_t delim = 0;
  const uint8_t *queries = nullptr, *db = nullptr;
  const int32_t *cutoffs = nullptr, *triggers = nullptr;
  const int32_t *matrix = nullptr;
  uint32_t number_letters = 0;
};

extern "C" int gzb_ungapped_extender_create(gzb_ungapped_extender **out) {
  GZB_CHECK(out, GZB_ERR_INVALID, "null output handle");
  *out = new (std::nothrow) gzb_ungapped_extender();
  GZB_CHECK(*out, GZB_ERR_NOMEM, "host allocation failed");
  return GZB_OK;
}
extern "C" int gzb_ungapped_extender_destroy(gzb_ungapped_extender *h) {
  delete h;
  return GZB_OK;
}
extern "C" int gzb_ungapped_extender_set_query_seed_data_list(
    gzb_ungapped_extender *h, const uint32_t *qid, const uint32_t *qpos) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->list_qid = qid;
  h->list_qpos = qpos;
  return GZB_OK;
}
extern "C" int gzb_ungapped_extender_set_queries(gzb_ungapped_extender *h,
                                                 uint8_t delim, const uint8_t *q,
                                                 const int32_t *cut,
                                                 const int32_t *trig) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->delim = delim;
  h->queries = q;
  h->cutoffs = cut;
  h->triggers = trig;
  return GZB_OK;
}
extern "C" int gzb_ungapped_extender_set_database(gzb_ungapped_extender *h,
                                                  const uint8_t *d) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->db = d;
  return GZB_OK;
}
extern "C" int gzb_ungapped_extender_set_score_matrix(gzb_ungapped_extender *h,
                                                      const int32_t *m,
                                                      uint32_t number_letters) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  GZB_CHECK(number_letters > 0 && number_letters < 32, GZB_ERR_INVALID,
            "number_letters %u out of range", number_letters);
  h->matrix = m;
  h->number_letters = number_letters;
  return GZB_OK;
}

static constexpr int kScanB = 256;

extern "C" size_t gzb_ungapped_extender_query_seeds_temp_bytes(size_t size) {
  size_t tiles = (size + kScanB - 1) / kScanB;
  size_t tiles2 = (tiles + kScanB - 1) / kScanB;
  return 4 * (tiles + tiles2 + 64);
}

// in-place inclusive max-scan over n elements using `tmp` (from
// gzb_ungapped_extender_query_seeds_temp_bytes)
static int max_scan(uint32_t *a, size_t n, uint32_t *tmp, cudaStream_t s, int depth = 0) {
  if (n == 0) return GZB_OK;
  const size_t tiles = (n + kScanB - 1) / kScanB;
  GZB_CHECK(tiles < (1u << 31) && depth < 4, GZB_ERR_OVERFLOW, "scan too large");
  max_scan_tiles<kScanB><<<(unsigned)tiles, kScanB, 0, s>>>(a, n, tmp);
  GZB_CUDA(cudaGetLastError());
  if (tiles > 1) {
    GZB_TRY(max_scan(tmp, tiles, tmp + tiles, s, depth + 1));
    max_scan_apply<kScanB><<<(unsigned)tiles, kScanB, 0, s>>>(a, n, tmp);
    GZB_CUDA(cudaGetLastError());
  }
  return GZB_OK;
}

extern "C" int gzb_ungapped_extender_set_query_seeds(
    gzb_ungapped_extender *h, size_t nseeds, size_t size, const uint32_t *seed_ids,
    const uint32_t *seed_starts, size_t temp_bytes, void *d_temp,
    uint32_t *d_seed_ids, uint32_t *d_seed_starts, uint32_t *d_qid,
    uint32_t *d_qpos, uint32_t *temp_array, void *stream) {
  GZB_CHECK(h && h->list_qid && h->list_qpos, GZB_ERR_INVALID,
            "query seed data list not set");
  if (size == 0) return GZB_OK;
  GZB_CHECK(temp_bytes >= gzb_ungapped_extender_query_seeds_temp_bytes(size),
            GZB_ERR_INVALID, "temp storage too small");
  cudaStream_t s = (cudaStream_t)stream;
  if (seed_starts)
    GZB_CUDA(cudaMemcpyAsync(d_seed_starts, seed_starts, 4 * nseeds, cudaMemcpyDefault, s));
  GZB_CUDA(cudaMemsetAsync(d_qid, 0, 4 * size, s));
  scatter_starts_kernel<<<grid_for(nseeds, 256), 256, 0, s>>>(nseeds, d_seed_starts, size, d_qid);
  GZB_CUDA(cudaGetLastError());
  GZB_CUDA(cudaMemcpyAsync(temp_array, d_qid, 4 * size, cudaMemcpyDeviceToDevice, s));
  GZB_TRY(max_scan(temp_array, size, (uint32_t *)d_temp, s));
  if (seed_ids)
    GZB_CUDA(cudaMemcpyAsync(d_seed_ids, seed_ids, 4 * nseeds, cudaMemcpyDefault, s));
  set_query_seeds_kernel<<<grid_for(size, 256), 256, 0, s>>>(
      size, h->list_qid, h->list_qpos, d_seed_ids, temp_array, d_qid, d_qpos);
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}

extern "C" int gzb_ungapped_extender_extend_with_trigger_async(
    gzb_ungapped_extender *h, size_t size, const uint32_t *qid, const uint32_t *qpos,
    const uint32_t *dpos, int8_t *flags, uint32_t *d_qid, uint32_t *d_qpos,
    uint32_t *d_dpos, int8_t *d_flags, int32_t *d_temp, void *stream) {
  (void)d_temp;
  GZB_CHECK(h && h->queries && h->db && h->matrix && h->cutoffs && h->triggers,
            GZB_ERR_INVALID, "ungapped extender not set up");
  if (size == 0) return GZB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (qid) GZB_CUDA(cudaMemcpyAsync(d_qid, qid, 4 * size, cudaMemcpyDefault, s));
  if (qpos) GZB_CUDA(cudaMemcpyAsync(d_qpos, qpos, 4 * size, cudaMemcpyDefault, s));
  if (dpos) GZB_CUDA(cudaMemcpyAsync(d_dpos, dpos, 4 * size, cudaMemcpyDefault, s));
  ungapped_trigger_kernel<<<grid_for(size, 256), 256, 0, s>>>(
      h->queries, h->db, h->delim, h->matrix, (int)h->number_letters,
      (int)h->number_letters + 1, h->cutoffs, h->triggers, size, d_qid, d_qpos, d_dpos,
      d_flags);
  GZB_CUDA(cudaGetLastError());
  if (flags) GZB_CUDA(cudaMemcpyAsync(flags, d_flags, size, cudaMemcpyDefault, s));
  return GZB_OK;
}

// --------------------------------------------------------------------------
// GappedExtenderGpu

struct gzb_gapped_extender {
  uint8_t delim = 0;
  const uint8_t *queries = nullptr, *db = nullptr;
  const int32_t *matrix = nullptr;
  uint32_t number_letters = 0;
  int gap_open = 0, gap_ext = 0, cutoff = 0;
  // device scratch: spill list, counters, fallback bands
  uint32_t *spill = nullptr;
  size_t spill_cap = 0;
  uint32_t *counters = nullptr;  // [0] spill count [1] too long
  unsigned long long *cells = nullptr;
  int2 *band_pool = nullptr;
  int band_wmask = 0;
  int serial_threads = 0;
};


extern "C" int gzb_gapped_extender_create(gzb_gapped_extender **out) {
  GZB_CHECK(out, GZB_ERR_INVALID, "null output handle");
  gzb_gapped_extender *h = new (std::nothrow) gzb_gapped_extender();
  GZB_CHECK(h, GZB_ERR_NOMEM, "host allocation failed");
  cudaError_t e = cudaMalloc(&h->counters, 64);
  if (e == cudaSuccess) e = cudaMalloc(&h->cells, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(h->counters, 0, 64);
  if (e == cudaSuccess) e = cudaMemset(h->cells, 0, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    cudaFree(h->counters);
    cudaFree(h->cells);
    delete h;
    return cuda_error(e, "gapped extender scratch", __FILE__, __LINE__);
  }
  *out = h;
  return GZB_OK;
}

extern "C" int gzb_gapped_extender_destroy(gzb_gapped_extender *h) {
  if (!h) return GZB_OK;
  cudaFree(h->spill);
  cudaFree(h->counters);
  cudaFree(h->cells);
  cudaFree(h->band_pool);
  delete h;
  return GZB_OK;
}
extern "C" int gzb_gapped_extender_set_queries(gzb_gapped_extender *h, uint8_t delim,
                                               const uint8_t *q) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->delim = delim;
  h->queries = q;
  return GZB_OK;
}
extern "C" int gzb_gapped_extender_set_database(gzb_gapped_extender *h,
                                                const uint8_t *d) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  h->db = d;
  return GZB_OK;
}
extern "C" int gzb_gapped_extender_set_score_parameters(gzb_gapped_extender *h,
                                                        const int32_t *m, uint32_t nl,
                                                        int open, int ext, int cutoff) {
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  GZB_CHECK(nl > 0 && nl < 32, GZB_ERR_INVALID, "number_letters %u out of range", nl);
  GZB_CHECK(open >= 0 && ext >= 0, GZB_ERR_INVALID, "negative gap penalty");
  h->matrix = m;
  h->number_letters = nl;
  h->gap_open = open;
  h->gap_ext = ext;
  h->cutoff = cutoff;
  return GZB_OK;
}

extern "C" int gzb_gapped_extender_convert_to_gapped_extension_seeds_async(
    gzb_gapped_extender *h, size_t size, int reverse, const uint32_t *seed_positions,
    const uint32_t *qpos, const uint32_t *dpos, uint32_t *d_seed_positions,
    uint32_t *d_temp, uint32_t *d_qpos, uint32_t *d_dpos, void *stream) {
  (void)reverse;
  GZB_CHECK(h, GZB_ERR_INVALID, "null handle");
  if (size == 0) return GZB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  GZB_CUDA(cudaMemcpyAsync(d_seed_positions, seed_positions, 4 * size, cudaMemcpyDefault, s));
  GZB_CUDA(cudaMemcpyAsync(d_temp, qpos, 4 * size, cudaMemcpyDefault, s));
  gather_kernel<<<grid_for(size, 256), 256, 0, s>>>(size, d_seed_positions, d_temp, d_qpos);
  GZB_CUDA(cudaGetLastError());
  GZB_CUDA(cudaMemcpyAsync(d_temp, dpos, 4 * size, cudaMemcpyDefault, s));
  gather_kernel<<<grid_for(size, 256), 256, 0, s>>>(size, d_seed_positions, d_temp, d_dpos);
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}

namespace gzb {
// Runs the three-level gapped extension over `n` extensions (optionally in
// the order given by `order`) whose positions sit in d_qpos/d_dpos (updated
// in place), writing d_scores (and each extension's DP cells to cells_out,
// if given, UINT32_MAX for those the thread kernel handed on).  The first
// level is the thread kernel `tile` names.  counters: [0] spilled from the thread
// kernel, [1] spilled from the warp kernel, [2] too long for the fallback.
// `spill` needs room for 2n entries.  Synchronises `s` once at the end.
// the serial fallback's band pool (allocated once)
int ensure_band_pool(int2 **band_pool, int *band_wmask) {
  if (!*band_pool) {
    GZB_CUDA(cudaMalloc(band_pool, sizeof(int2) * (size_t)kSerialThreads * kSerialBand));
    *band_wmask = kSerialBand - 1;
  }
  return GZB_OK;
}

int run_gapped(const GappedTile &tile, const GappedJob &job, const int32_t *matrix,
               int number_letters, int stride, size_t n, const uint32_t *order, int reverse,
               const uint8_t *dir, uint32_t *d_qpos, uint32_t *d_dpos, int32_t *d_scores,
               uint32_t **spill, size_t *spill_cap, uint32_t *counters,
               unsigned long long *cells, uint32_t *cells_out, int2 **band_pool,
               int *band_wmask, cudaStream_t s, uint32_t *n_fallback, const uint64_t *n_dev) {
  // n_dev: the count is read on the device (n bounds it and sizes the
  // grids), and the spill counts are left in counters for the caller (no
  // host synchronisation)
  if (n == 0) return GZB_OK;
  if (*spill_cap < 2 * n) {
    cudaFree(*spill);
    *spill = nullptr;
    *spill_cap = 0;
    GZB_CUDA(cudaMalloc(spill, 4 * 2 * n));
    *spill_cap = 2 * n;
  }
  GZB_TRY(ensure_band_pool(band_pool, band_wmask));
  GZB_CUDA(cudaMemsetAsync(counters, 0, 16, s));
  uint32_t *spill1 = *spill, *spill2 = *spill + n;
  // counters[0..3]: spill counts; counters[8..9]: the work queue (64-bit)
  GZB_TRY(launch_gapped_thread(tile, job, matrix, number_letters, stride, n, order,
                               (unsigned long long *)(counters + 8), reverse, dir, d_qpos,
                               d_dpos, d_scores, spill1, counters, cells, cells_out, s, n_dev));
  const uint32_t *serial_list = spill1, *serial_count = counters;
  if (warp_path_exact(job.cutoff)) {
    gapped_warp_kernel<<<148 * 4, kGappedWarps * 32, 0, s>>>(
        job, matrix, number_letters, stride, spill1, counters, reverse, dir, d_qpos, d_dpos,
        d_scores, spill2, counters + 1, cells);
    GZB_CUDA(cudaGetLastError());
    serial_list = spill2;
    serial_count = counters + 1;
  }
  gapped_serial_kernel<<<kSerialThreads / 128, 128, 0, s>>>(
      job, matrix, number_letters, stride, serial_list, serial_count, reverse, dir, d_qpos,
      d_dpos, d_scores, *band_pool, *band_wmask, cells, counters + 2);
  GZB_CUDA(cudaGetLastError());
  if (n_dev) return GZB_OK;
  uint32_t h[3] = {0, 0, 0};
  GZB_CUDA(cudaMemcpyAsync(h, counters, 12, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  GZB_CHECK(h[2] == 0, GZB_ERR_OVERFLOW,
            "%u gapped extensions need a band wider than %d columns", h[2], kSerialBand);
  if (n_fallback) *n_fallback = h[0];
  return GZB_OK;
}
}  // namespace gzb

extern "C" int gzb_gapped_extender_extend_one_side_score_only_async(
    gzb_gapped_extender *h, size_t size, int reverse, uint32_t *qpos, uint32_t *dpos,
    int32_t *scores, uint32_t *d_qpos, uint32_t *d_dpos, int32_t *d_scores,
    void *stream) {
  GZB_CHECK(h && h->queries && h->db && h->matrix, GZB_ERR_INVALID,
            "gapped extender not set up");
  if (size == 0) return GZB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  GappedJob job;
  job.query = h->queries;
  job.db = h->db;
  job.delim = h->delim;
  job.gap_open = h->gap_open;
  job.gap_ext = h->gap_ext;
  job.cutoff = h->cutoff;
  GZB_TRY(run_gapped(g_tile, job, h->matrix, (int)h->number_letters,
                     (int)h->number_letters + 1, size, nullptr, reverse, nullptr, d_qpos,
                     d_dpos, d_scores, &h->spill, &h->spill_cap, h->counters, h->cells, nullptr,
                     &h->band_pool, &h->band_wmask, s, nullptr, nullptr));
  if (qpos) GZB_CUDA(cudaMemcpyAsync(qpos, d_qpos, 4 * size, cudaMemcpyDefault, s));
  if (dpos) GZB_CUDA(cudaMemcpyAsync(dpos, d_dpos, 4 * size, cudaMemcpyDefault, s));
  if (scores) GZB_CUDA(cudaMemcpyAsync(scores, d_scores, 4 * size, cudaMemcpyDefault, s));
  return GZB_OK;
}

extern "C" int gzb_gapped_extender_cells(gzb_gapped_extender *h, uint64_t *cells) {
  GZB_CHECK(h && cells, GZB_ERR_INVALID, "null argument");
  unsigned long long c = 0;
  GZB_CUDA(cudaMemcpy(&c, h->cells, sizeof(c), cudaMemcpyDeviceToHost));
  *cells = c;
  return GZB_OK;
}

namespace gzb {
int check_tile_value(int which, int value) {
  if (which == GZB_TILE_GAPPED_KERNEL) {
    GZB_CHECK(value >= GZB_GAPPED_KERNEL_FLAT && value <= GZB_GAPPED_KERNEL_GROUP32,
              GZB_ERR_INVALID,
              "gapped kernel %d is none of GZB_GAPPED_KERNEL_FLAT/LANE/ROWS/STATIC/DEAL/GROUP*",
              value);
    return GZB_OK;
  }
  if (which == GZB_TILE_ORDER) {
    GZB_CHECK(value == GZB_ORDER_HITS || value == GZB_ORDER_MODEL, GZB_ERR_INVALID,
              "order %d is neither GZB_ORDER_HITS nor GZB_ORDER_MODEL", value);
    return GZB_OK;
  }
  if (which == GZB_TILE_SEED_WALKER) {
    GZB_CHECK(value == GZB_SEED_WALKER_UNIT || value == GZB_SEED_WALKER_DEALT, GZB_ERR_INVALID,
              "seed walker %d is neither GZB_SEED_WALKER_UNIT nor GZB_SEED_WALKER_DEALT", value);
    return GZB_OK;
  }
  if (which == GZB_TILE_BAND_WIDTH) {
    GZB_CHECK(value == 32 || value == 64 || value == 128, GZB_ERR_INVALID,
              "band width %d is none of 32, 64, 128", value);
    return GZB_OK;
  }
  GZB_CHECK(which == GZB_TILE_BOOK_THRESHOLD, GZB_ERR_INVALID, "unknown tile parameter %d", which);
  GZB_CHECK(value >= 1 && value <= 32, GZB_ERR_INVALID, "book threshold %d outside 1..32", value);
  return GZB_OK;
}
int *tile_field(GappedTile &t, int which) {
  return which == GZB_TILE_GAPPED_KERNEL ? &t.kernel
         : which == GZB_TILE_ORDER      ? &t.order
         : which == GZB_TILE_SEED_WALKER ? &t.seed_walker
         : which == GZB_TILE_BAND_WIDTH  ? &t.band_width
                                        : &t.book_threshold;
}
// a valid value of tile parameter `which` (for checking `which` alone)
int any_tile_value(int which) {
  return which == GZB_TILE_GAPPED_KERNEL ? GZB_GAPPED_KERNEL_FLAT
         : which == GZB_TILE_ORDER      ? GZB_ORDER_HITS
         : which == GZB_TILE_SEED_WALKER ? GZB_SEED_WALKER_UNIT
         : which == GZB_TILE_BAND_WIDTH  ? kLaneW
                                        : 1;
}
}  // namespace gzb

extern "C" int gzb_set_tile_parameter(int which, int value) {
  GZB_TRY(gzb::check_tile_value(which, value));
  *gzb::tile_field(gzb::g_tile, which) = value;
  return GZB_OK;
}

extern "C" int gzb_get_tile_parameter(int which, int *value) {
  GZB_CHECK(value, GZB_ERR_INVALID, "null value");
  GZB_TRY(gzb::check_tile_value(which, gzb::any_tile_value(which)));
  *value = *gzb::tile_field(gzb::g_tile, which);
  return GZB_OK;
}
