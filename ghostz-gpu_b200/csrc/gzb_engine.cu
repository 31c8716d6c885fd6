// gzb_engine.cu -- device-resident presearch of one database chunk.
//
// Stage map (reference functions in parentheses):
//   set_database : seed index with subsequence clustering, built on the device
//                  (SeedSearcherDatabaseParameters::Build,
//                   src/seed_searcher_database_parameters.cpp:41-319)
//   set_queries  : query hash lists
//                  (SeedSearcherGpuQueryParameters::Build,
//                   src/seed_searcher_gpu_query_parameters.cpp:17-272)
//   presearch    : seed search + distance filter + ungapped X-drop with
//                  trigger, fused (SeedSearcherGpu::Search*,
//                  src/seed_searcher_gpu.cpp:186-537; DistanceCalculatorGpu;
//                  UngappedExtenderGpu::ExtendWithTriggerAsync)
//                  -> chain filter (ChainFilter::Filter, src/chain_filter.cpp:24-99)
//                  -> gapped X-drop both sides (GappedExtenderGpu)
//                  -> top-b merge (AlignerCommon::AddResults,
//                     src/aligner_common.h:147-274)
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "ghostz_b200.h"
#include "gzb_blob.h"
#include "gzb_common.h"
#include "gzb_index.cuh"
#include "gzb_kernels.cuh"
#include "gzb_cost.cuh"
#include "gzb_traceback.cuh"

namespace cg = cooperative_groups;

namespace gzb {

int cost_predict(const float *d_params, const float *d_x, uint32_t n, float *d_out,
                 cudaStream_t s, const uint64_t *n_dev);
int cost_train(const float *d_x, const float *d_y, uint32_t n, float *params, int epochs,
               int batch, float lr, uint64_t seed, float *final_loss, cudaStream_t s);
__global__ void gapped_warp_kernel(GappedJob job, const int32_t *__restrict__ matrix,
                                   int number_letters, int stride, const uint32_t *list,
                                   const uint32_t *list_count, int reverse,
                                   const uint8_t *__restrict__ dir, uint32_t *qpos,
                                   uint32_t *dpos, int32_t *scores, uint32_t *spill,
                                   uint32_t *spill_count, unsigned long long *cells_total);
__global__ void gapped_serial_kernel(GappedJob job, const int32_t *__restrict__ matrix,
                                     int number_letters, int stride, const uint32_t *list,
                                     const uint32_t *list_count, int reverse,
                                     const uint8_t *__restrict__ dir, uint32_t *qpos,
                                     uint32_t *dpos, int32_t *scores, int2 *band_pool,
                                     int wmask, unsigned long long *cells_total,
                                     uint32_t *too_long_count);

extern GappedTile g_tile;
constexpr int kTileParameters = 5;  // GZB_TILE_BOOK_THRESHOLD .. GZB_TILE_BAND_WIDTH
int check_tile_value(int which, int value);
int *tile_field(GappedTile &t, int which);
int any_tile_value(int which);
int ensure_band_pool(int2 **band_pool, int *band_wmask);
int run_gapped(const GappedTile &tile, const GappedJob &job, const int32_t *matrix,
               int number_letters, int stride, size_t n, const uint32_t *order, int reverse,
               const uint8_t *dir, uint32_t *d_qpos, uint32_t *d_dpos, int32_t *d_scores,
               uint32_t **spill, size_t *spill_cap, uint32_t *counters,
               unsigned long long *cells, uint32_t *cells_out, int2 **band_pool,
               int *band_wmask, cudaStream_t s, uint32_t *n_fallback, const uint64_t *n_dev);

constexpr uint64_t kPad = 256;  // delimiter bytes kept around device sequences

// Growable device buffer.
struct DBuf {
  void *p = nullptr;
  size_t bytes = 0;
  int ensure(size_t need) {
    if (need <= bytes) return GZB_OK;
    cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t n = need + need / 4 + 256;
    GZB_CUDA(cudaMalloc(&p, n));
    bytes = n;
    return GZB_OK;
  }
  void release() {
    cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T *as() const {
    return (T *)p;
  }
};

static unsigned grid1(uint64_t n, int block, unsigned cap = 148u * 32u) {
  uint64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// ---------------------------------------------------------------------------
// warp-aggregated append (ballot compaction)
template <class T>
__device__ __forceinline__ void append(T *buf, unsigned long long *count,
                                       unsigned long long cap, const T &v) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(count, (unsigned long long)g.size());
  base = g.shfl(base, 0);
  const unsigned long long slot = base + g.thread_rank();
  if (slot < cap) buf[slot] = v;
}

__device__ __forceinline__ void add_counter(unsigned long long *c, unsigned long long v) {
  v += __shfl_down_sync(0xffffffffu, v, 16);
  v += __shfl_down_sync(0xffffffffu, v, 8);
  v += __shfl_down_sync(0xffffffffu, v, 4);
  v += __shfl_down_sync(0xffffffffu, v, 2);
  v += __shfl_down_sync(0xffffffffu, v, 1);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(c, v);
}

// ---------------------------------------------------------------------------
// database index kernels

// Keep rule of the index build (:85-108): a k-mer is dropped when the next
// position's k-mer is contained in it.
__global__ void db_pairs_kernel(DevParams p, const uint8_t *__restrict__ db, uint64_t len,
                                uint64_t *pairs, unsigned long long *count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t h, h2;
    int hl, hl2;
    if (!seed_hash(p, db + i, &h, &hl)) continue;
    if (i + 1 < len && seed_hash(p, db + i + 1, &h2, &hl2) && hl2 + 1 <= hl) continue;
    append(pairs, count, len, ((uint64_t)h << 32) | (uint64_t)i);
  }
}

// Per sorted entry: bucket start flag, non-clustering state and the packed
// similarity window (4 bits per code).
__global__ void db_entry_kernel(DevParams p, const uint8_t *__restrict__ db,
                                const uint64_t *__restrict__ pairs, uint64_t n,
                                uint8_t *flag_start, uint8_t *state, uint64_t *window) {
  const int L = p.subsequence_length, half = L / 2;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = pairs[i];
    flag_start[i] = (i == 0 || (pairs[i - 1] >> 32) != (k >> 32)) ? 1 : 0;
    const uint32_t c = (uint32_t)k;
    uint8_t st = 0;
    uint64_t w = 0;
    if ((int)c < half) {
      st = 1;
    } else {
      for (int t = 0; t < L; ++t) {
        const int x = db[c - half + t];
        if (x == p.delimiter) {
          st = 1;
          break;
        }
        w |= (uint64_t)(p.sim_map[x] & 15) << (4 * t);
      }
    }
    state[i] = st;
    window[i] = w;
  }
}

// Greedy clustering inside each hash bucket (:117-205): walking the bucket
// in position order, every still-free entry becomes a representative and
// claims the later free entries within max_member_distance mismatches.
// One warp per bucket.
__global__ void cluster_kernel(const uint32_t *__restrict__ bucket_start, uint64_t n_buckets,
                               uint64_t n, uint8_t *state, const uint64_t *__restrict__ window,
                               uint32_t *rep_of, int max_mismatch) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t b = warp; b < n_buckets; b += nwarps) {
    const uint64_t s = bucket_start[b];
    const uint64_t e = (b + 1 < n_buckets) ? bucket_start[b + 1] : n;
    if (e - s < 2) {
      if (lane == 0 && state[s] == 0) state[s] = 2;
      continue;
    }
    for (uint64_t i = s; i < e; ++i) {
      const uint8_t st = state[i];  // uniform: written before the last __syncwarp
      if (st != 0) continue;
      const uint64_t wr = window[i];
      if (lane == 0) state[i] = 2;
      for (uint64_t j = i + 1 + lane; j < e; j += 32) {
        if (state[j] == 0 && nibble_mismatches(wr, window[j]) <= max_mismatch) {
          state[j] = 3;
          rep_of[j] = (uint32_t)i;
        }
      }
      __syncwarp();
    }
  }
}

__global__ void member_count_kernel(const uint8_t *state, const uint32_t *rep_of, uint64_t n,
                                    uint32_t *member_count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (state[i] == 3) atomicAdd(&member_count[rep_of[i]], 1u);
}

// class flags: nc (0/1), rep (0/1)
__global__ void classify_kernel(const uint8_t *state, const uint32_t *member_count, uint64_t n,
                                uint8_t *is_nc, uint8_t *is_rep, uint8_t *is_member) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const bool rep = state[i] == 2 && member_count[i] > 0;
    const bool mem = state[i] == 3;
    is_rep[i] = rep;
    is_member[i] = mem;
    is_nc[i] = !rep && !mem;
  }
}

__global__ void key_start_flags(const uint64_t *keys, uint64_t n, uint8_t *flag) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || (keys[i - 1] >> 32) != (keys[i] >> 32)) ? 1 : 0;
}

__global__ void iota_u32(uint32_t *a, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = (uint32_t)i;
}

// keys/offsets/values of a CSR from hash-sorted (hash<<32|value) pairs and
// the indices of segment starts.
__global__ void csr_fill(const uint64_t *pairs, uint64_t n, const uint32_t *starts,
                         uint64_t nseg, uint32_t *keys, uint32_t *offsets, uint32_t *values) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    values[i] = (uint32_t)pairs[i];
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s <= nseg;
       s += (uint64_t)gridDim.x * blockDim.x) {
    if (s < nseg) {
      keys[s] = (uint32_t)(pairs[starts[s]] >> 32);
      offsets[s] = starts[s];
    } else {
      offsets[s] = (uint32_t)n;
    }
  }
}

// rank of each representative entry = its cluster id
__global__ void scatter_cluster_ids(const uint32_t *rep_entries, uint64_t nrep,
                                    uint32_t *cid_of_entry, uint32_t *cluster_ids) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < nrep;
       r += (uint64_t)gridDim.x * blockDim.x) {
    cid_of_entry[rep_entries[r]] = (uint32_t)r;
    cluster_ids[r] = (uint32_t)r;
  }
}

__global__ void member_pairs_kernel(const uint32_t *member_entries, uint64_t nm,
                                    const uint32_t *rep_of, const uint32_t *cid_of_entry,
                                    const uint64_t *pairs, uint64_t *out, uint32_t *cnt) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nm;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t e = member_entries[i];
    const uint32_t cid = cid_of_entry[rep_of[e]];
    out[i] = ((uint64_t)cid << 32) | (uint32_t)pairs[e];
    atomicAdd(&cnt[cid], 1u);
  }
}

__global__ void low32(const uint64_t *in, uint64_t n, uint32_t *out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)in[i];
}

// ---------------------------------------------------------------------------
// query lists

// One warp per query, a lane per position: every position of a
// delimiter-free stretch of at least L residues is hashed; key = hash<<32 |
// nocheck<<31 | concat pos.  A position's stretch is bounded by its nearest
// delimiters (prev, next: delim_dist_kernel); keys are appended warp-wide.
__global__ void query_entries_kernel(DevParams p, const uint8_t *__restrict__ q,
                                     const uint32_t *__restrict__ offsets,
                                     const uint32_t *__restrict__ lengths,
                                     const uint32_t *__restrict__ prev,
                                     const uint32_t *__restrict__ next, uint32_t nq,
                                     uint64_t *keys, unsigned long long *count,
                                     unsigned long long cap) {
  const uint32_t L = (uint32_t)p.subsequence_length;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t qi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; qi < nq; qi += warps) {
    const uint32_t base = offsets[qi], len = lengths[qi];
    for (uint32_t i0 = 0; i0 < len; i0 += 32) {
      const uint32_t i = i0 + lane;
      const uint32_t pos = base + i;
      bool have = false;
      uint64_t k = 0;
      if (i < len && q[pos] != p.delimiter) {
        const uint32_t off = prev[pos] + 1 - base, end = next[pos] - base;  // the stretch
        uint32_t h;
        int hl;
        if (end - off >= L && seed_hash(p, q + pos, &h, &hl)) {
          const uint32_t cs = off + L / 2, ce = end - L / 2;
          const uint64_t nocheck = (cs <= i && i < ce) ? 0 : 1;
          k = ((uint64_t)h << 32) | (nocheck << 31) | (uint64_t)pos;
          have = true;
        }
      }
      if (have) append(keys, count, cap, k);
    }
  }
}

// lists from sorted entry keys: per list hash, offset and check count;
// per entry the query id and concatenated position
__global__ void list_fill_kernel(const uint64_t *keys, uint64_t n, const uint32_t *starts,
                                 uint64_t nl, const uint32_t *q_offsets, uint32_t nq,
                                 uint32_t *hash, uint32_t *offsets, uint32_t *nchk,
                                 uint32_t *entry_qid, uint32_t *entry_cpos) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t cpos = (uint32_t)(keys[i] & 0x7fffffffu);
    // query: largest qi with offsets[qi] <= cpos
    uint32_t lo = 0, hi = nq - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (q_offsets[mid] <= cpos)
        lo = mid;
      else
        hi = mid - 1;
    }
    entry_qid[i] = lo;
    entry_cpos[i] = cpos;
  }
  for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l <= nl;
       l += (uint64_t)gridDim.x * blockDim.x) {
    if (l == nl) {
      offsets[l] = (uint32_t)n;
      continue;
    }
    const uint32_t b = starts[l];
    const uint32_t e = (l + 1 < nl) ? starts[l + 1] : (uint32_t)n;
    hash[l] = (uint32_t)(keys[b] >> 32);
    offsets[l] = b;
    // check entries (nocheck bit 0) come first
    uint32_t lo = b, hi = e;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (((keys[mid] >> 31) & 1) == 0)
        lo = mid + 1;
      else
        hi = mid;
    }
    nchk[l] = lo - b;
  }
}

// per entry: the packed similarity window and the query's ungapped cutoff
// and trigger (cutoff << 16 | trigger as int16; both checked to fit)
__global__ void entry_window_kernel(DevParams p, const uint8_t *__restrict__ q,
                                    const uint32_t *__restrict__ cpos,
                                    const uint32_t *__restrict__ qid,
                                    const int32_t *__restrict__ cutoffs,
                                    const int32_t *__restrict__ triggers, uint64_t n,
                                    uint64_t *out, uint32_t *ct) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    out[i] = pack_window(p, q + cpos[i]);
    const uint32_t id = qid[i];
    ct[i] = ((uint32_t)cutoffs[id] << 16) | (uint32_t)(uint16_t)(int16_t)triggers[id];
  }
}

__global__ void list_lookup_kernel(DevLists L, DevIndex X, int clustering,
                                   uint64_t *unit_counts) {
  for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < L.n_lists;
       l += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t h = L.hash[l];
    uint32_t rb = 0, rc = 0, nb = 0, nc = 0;
    if (clustering) {
      const long long r = find_key(X.rep_keys, X.n_rep_keys, h);
      if (r >= 0) {
        rb = X.rep_offsets[r];
        rc = X.rep_offsets[r + 1] - rb;
      }
    }
    const long long v = find_key(X.nc_keys, X.n_nc_keys, h);
    if (v >= 0) {
      nb = X.nc_offsets[v];
      nc = X.nc_offsets[v + 1] - nb;
    }
    L.rep_begin[l] = rb;
    L.rep_count[l] = rc;
    L.nc_begin[l] = nb;
    L.nc_count[l] = nc;
    unit_counts[l] = (uint64_t)rc + nc;  // exclusive-scanned into unit_offsets
  }
}

// ---------------------------------------------------------------------------
// presearch kernels

struct SeedArgs {
  DevParams p;
  DevLists L;
  DevIndex X;
  const uint8_t *q;
  const uint8_t *db;
  const uint32_t *q_offsets;
  const int32_t *cutoffs;
  const int32_t *triggers;
  const int32_t *matrix32;  // 32x32
  int clustering;
  int dbits, qbits;         // packed hit key: qid | d << qbits | q
  uint64_t *hits;
  unsigned long long *hit_count;
  unsigned long long hit_cap;
  uint2 *mwork;             // member work: (cluster id, entry index)
  unsigned long long *mwork_count;
  unsigned long long mwork_cap;
  unsigned long long *ctr;  // [0] distance seeds [1] ungapped seeds [2] steps
  const uint64_t *units_dev = nullptr;  // unit count on the device (else L.n_units)
};

__device__ __forceinline__ void emit_hit(const SeedArgs &a, uint32_t qid, uint32_t d,
                                         uint32_t qp) {
  const uint64_t key = ((uint64_t)qid << (a.dbits + a.qbits)) |
                       ((uint64_t)d << a.qbits) | (uint64_t)qp;
  append(a.hits, a.hit_count, a.hit_cap, key);
}

constexpr int kSeedBlock = 256;
constexpr int kUnitsPerWarp = 256;

// One unit = one representative or one residual database position of a list,
// tried against every query position of that list.  Bounded to six blocks
// per SM (40 registers, a few spilled): the walks' global loads want the
// warps more than the registers.
__global__ void __launch_bounds__(kSeedBlock, 6)
seed_kernel(SeedArgs a) {
  __shared__ __align__(16) int32_t tbl32[kWalkTableBytes / 4];
  load_walk_table(tbl32, a.matrix32, a.p.delimiter);
  __syncthreads();
  const char *tbl = reinterpret_cast<const char *>(tbl32);
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t U = a.units_dev ? *a.units_dev : a.L.n_units;
  const int thr = a.p.distance_threshold;
  const int maxmd = a.p.max_member_distance;
  // a thread's counts stay far below 2^32 (that many walk steps would take
  // one thread seconds); 32-bit counters leave the six-block register
  // budget to the walk
  uint32_t n_dist = 0, n_seed = 0, n_steps = 0;
  for (uint64_t base = warp * kUnitsPerWarp; base < U; base += nwarps * kUnitsPerWarp) {
    const uint64_t last = min(base + kUnitsPerWarp, U) - 1;
    // list range of this warp's units
    uint64_t l_lo = 0, l_hi = 0;
    if (lane == 0) {
      l_lo = upper_segment(a.L.unit_offsets, 0, a.L.n_lists - 1, base);
      l_hi = upper_segment(a.L.unit_offsets, l_lo, a.L.n_lists - 1, last);
    }
    l_lo = __shfl_sync(0xffffffffu, l_lo, 0);
    l_hi = __shfl_sync(0xffffffffu, l_hi, 0);
    for (uint64_t u = base + lane; u <= last; u += 32) {
      const uint64_t l = upper_segment(a.L.unit_offsets, l_lo, l_hi, u);
      const uint32_t j = (uint32_t)(u - a.L.unit_offsets[l]);
      const uint32_t pb = a.L.offsets[l], pe = a.L.offsets[l + 1];
      const uint32_t nchk = a.L.nchk[l];
      const uint32_t nrep = a.L.rep_count[l];
      if (j < nrep) {
        // representative: distance filter for check positions
        const uint32_t r = a.L.rep_begin[l] + j;
        const uint32_t rpos = a.X.rep_positions[r];
        const uint32_t cid = a.X.rep_cluster_ids[r];
        const bool members = a.X.member_offsets[cid + 1] > a.X.member_offsets[cid];
        const uint64_t rwin = a.X.rep_windows[r];
        const uint8_t *dptr = a.db + rpos;
        for (uint32_t k = pb; k < pe; ++k) {
          const uint32_t cpos = a.L.entry_cpos[k];
          const uint8_t *qptr = a.q + cpos;
          bool try_rep, pass;
          if (k < pb + nchk) {
            const int dist = nibble_mismatches(a.L.entry_window[k], rwin);
            ++n_dist;
            try_rep = dist <= thr;
            pass = max(dist - maxmd, 0) <= thr;
          } else {
            try_rep = true;
            pass = true;
          }
          if (try_rep) {
            int steps = 0;
            ++n_seed;
            const uint32_t ct = a.L.entry_ct[k];
            if (walk_hit(qptr, dptr, tbl, (int)(ct >> 16), (int)(int16_t)(ct & 0xffffu),
                         &steps)) {
              const uint32_t qid = a.L.entry_qid[k];  // only a hit needs its query
              emit_hit(a, qid, rpos, cpos - a.q_offsets[qid]);
            }
            n_steps += steps;
          }
          if (pass && members) append(a.mwork, a.mwork_count, a.mwork_cap, make_uint2(cid, k));
        }
      } else {
        const uint32_t d = a.X.nc_values[a.L.nc_begin[l] + (j - nrep)];
        const uint8_t *dptr = a.db + d;
        for (uint32_t k = pb; k < pe; ++k) {
          const uint32_t cpos = a.L.entry_cpos[k];
          int steps = 0;
          ++n_seed;
          const uint32_t ct = a.L.entry_ct[k];
          if (walk_hit(a.q + cpos, dptr, tbl, (int)(ct >> 16), (int)(int16_t)(ct & 0xffffu),
                       &steps)) {
            const uint32_t qid = a.L.entry_qid[k];  // only a hit needs its query
            emit_hit(a, qid, d, cpos - a.q_offsets[qid]);
          }
          n_steps += steps;
        }
      }
    }
  }
  __syncwarp();
  add_counter(&a.ctr[0], n_dist);
  add_counter(&a.ctr[1], n_seed);
  add_counter(&a.ctr[2], n_steps);
}

// Members of a representative's cluster against one passing query position
// (one work item = (cluster id, list entry)).  Each warp loads 32 items
// together, scans their member counts, and deals the (item, member) seeds
// to its lanes 32 at a time: a lane finds its item with a five-step shuffle
// search over the scan, so a seed costs one load (the member's position)
// besides its walk.  Six blocks per SM, as seed_kernel.
__global__ void __launch_bounds__(kSeedBlock, 6)
member_kernel(SeedArgs a, const uint2 *__restrict__ mwork, uint64_t n_work,
              const uint64_t *n_dev) {
  __shared__ __align__(16) int32_t tbl32[kWalkTableBytes / 4];
  if (n_dev) n_work = *n_dev;
  load_walk_table(tbl32, a.matrix32, a.p.delimiter);
  __syncthreads();
  const char *tbl = reinterpret_cast<const char *>(tbl32);
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  uint32_t n_seed = 0, n_steps = 0;  // per thread, as in seed_kernel
  for (uint64_t i0 = warp * 32; i0 < n_work; i0 += nwarps * 32) {
    const uint64_t i = i0 + lane;
    uint32_t mb = 0, cnt = 0, qid = 0, cpos = 0, ct = 0;
    if (i < n_work) {
      const uint2 mw = mwork[i];
      mb = a.X.member_offsets[mw.x];
      cnt = a.X.member_offsets[mw.x + 1] - mb;
      qid = a.L.entry_qid[mw.y];
      cpos = a.L.entry_cpos[mw.y];
      ct = a.L.entry_ct[mw.y];
    }
    uint32_t incl = cnt;  // inclusive scan of member counts
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    const uint32_t excl = incl - cnt;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t p = base + lane;
      // owner: the last lane whose exclusive offset is <= p (it has p < its
      // inclusive offset, since every later lane starts beyond p)
      int o = 0;
      for (int step = 16; step >= 1; step >>= 1) {
        const uint32_t e = __shfl_sync(0xffffffffu, excl, o + step);
        if (o + step < 32 && e <= p) o += step;
      }
      const uint32_t m = __shfl_sync(0xffffffffu, mb, o) + (p - __shfl_sync(0xffffffffu, excl, o));
      const uint32_t sq = __shfl_sync(0xffffffffu, qid, o);
      const uint32_t sc = __shfl_sync(0xffffffffu, cpos, o);
      const uint32_t sct = __shfl_sync(0xffffffffu, ct, o);
      if (p < total) {
        const uint32_t d = a.X.member_positions[m];
        int steps = 0;
        ++n_seed;
        if (walk_hit(a.q + sc, a.db + d, tbl, (int)(sct >> 16), (int)(int16_t)(sct & 0xffffu),
                     &steps))
          emit_hit(a, sq, d, sc - a.q_offsets[sq]);
        n_steps += steps;
      }
    }
  }
  __syncwarp();
  add_counter(&a.ctr[1], n_seed);
  add_counter(&a.ctr[2], n_steps);
}

// ---------------------------------------------------------------------------
// Dealt seed walker.  seed_kernel gives each lane whole units (a unit's
// every list entry in turn), so a warp waits for its lane with the longest
// list.  Here the seeds of 32 units -- every (unit, list entry) pair -- form
// one stream that is dealt to the lanes 32 at a time, as member_kernel deals
// member seeds: a warp then waits only for the longest single walk of a
// round.  A lane finds its seed's unit with a shuffle search over the
// units' exclusive count scan.  Every seed gets the same decisions and
// counts as in seed_kernel.

constexpr unsigned kFullMask = 0xffffffffu;

// the last lane whose exclusive offset is <= p (the owner of stream seed p)
__device__ __forceinline__ int stream_owner(uint32_t excl, uint32_t p) {
  int o = 0;
  for (int step = 16; step >= 1; step >>= 1) {
    const uint32_t e = __shfl_sync(kFullMask, excl, (o + step) & 31);
    if (o + step < 32 && e <= p) o += step;
  }
  return o;
}

__global__ void __launch_bounds__(kSeedBlock, 4)
seed_dealt_kernel(SeedArgs a) {
  __shared__ __align__(16) int32_t tbl32[kWalkTableBytes / 4];
  load_walk_table(tbl32, a.matrix32, a.p.delimiter);
  __syncthreads();
  const char *tbl = reinterpret_cast<const char *>(tbl32);
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t U = a.units_dev ? *a.units_dev : a.L.n_units;
  const int thr = a.p.distance_threshold;
  const int maxmd = a.p.max_member_distance;
  unsigned long long n_dist = 0, n_seed = 0, n_steps = 0;
  for (uint64_t base = warp * kUnitsPerWarp; base < U; base += nwarps * kUnitsPerWarp) {
    const uint64_t last = min(base + kUnitsPerWarp, U) - 1;
    uint64_t l_lo = 0, l_hi = 0;
    if (lane == 0) {
      l_lo = upper_segment(a.L.unit_offsets, 0, a.L.n_lists - 1, base);
      l_hi = upper_segment(a.L.unit_offsets, l_lo, a.L.n_lists - 1, last);
    }
    l_lo = __shfl_sync(kFullMask, l_lo, 0);
    l_hi = __shfl_sync(kFullMask, l_hi, 0);
    for (uint64_t b0 = base; b0 <= last; b0 += 32) {
      // this lane's unit: database position, entry range, filter data
      const uint64_t u = b0 + lane;
      uint32_t cnt = 0, pb = 0, chk_end = 0, upos = 0, cid = 0;
      uint64_t rwin = 0;
      bool rep = false, members = false;
      if (u <= last) {
        const uint64_t l = upper_segment(a.L.unit_offsets, l_lo, l_hi, u);
        const uint32_t j = (uint32_t)(u - a.L.unit_offsets[l]);
        pb = a.L.offsets[l];
        cnt = a.L.offsets[l + 1] - pb;
        const uint32_t nrep = a.L.rep_count[l];
        if (j < nrep) {
          const uint32_t r = a.L.rep_begin[l] + j;
          rep = true;
          upos = a.X.rep_positions[r];
          cid = a.X.rep_cluster_ids[r];
          members = a.X.member_offsets[cid + 1] > a.X.member_offsets[cid];
          rwin = a.X.rep_windows[r];
          chk_end = pb + a.L.nchk[l];
        } else {
          upos = a.X.nc_values[a.L.nc_begin[l] + (j - nrep)];
        }
      }
      uint32_t incl = cnt;
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(kFullMask, incl, d);
        if (lane >= d) incl += t;
      }
      const uint32_t excl = incl - cnt;
      const uint32_t total = __shfl_sync(kFullMask, incl, 31);
      for (uint32_t r0 = 0; r0 < total; r0 += 32) {
        const uint32_t p = r0 + lane;
        const int o = stream_owner(excl, p < total ? p : 0);
        const uint32_t opb = __shfl_sync(kFullMask, pb, o);
        const uint32_t oexcl = __shfl_sync(kFullMask, excl, o);
        const uint32_t ochk = __shfl_sync(kFullMask, chk_end, o);
        const uint32_t opos = __shfl_sync(kFullMask, upos, o);
        const uint32_t ocid = __shfl_sync(kFullMask, cid, o);
        const uint64_t owin = __shfl_sync(kFullMask, rwin, o);
        const bool orep = __shfl_sync(kFullMask, rep, o);
        const bool omem = __shfl_sync(kFullMask, members, o);
        if (p < total) {
          const uint32_t k = opb + (p - oexcl);
          bool walk = true;
          if (orep) {
            bool pass = true;
            if (k < ochk) {
              const int dist = nibble_mismatches(a.L.entry_window[k], owin);
              ++n_dist;
              walk = dist <= thr;
              pass = max(dist - maxmd, 0) <= thr;
            }
            if (pass && omem) append(a.mwork, a.mwork_count, a.mwork_cap, make_uint2(ocid, k));
          }
          if (walk) {
            const uint32_t qid = a.L.entry_qid[k], cpos = a.L.entry_cpos[k];
            const uint32_t ct = a.L.entry_ct[k];
            int steps = 0;
            ++n_seed;
            if (walk_hit(a.q + cpos, a.db + opos, tbl, (int)(ct >> 16),
                         (int)(int16_t)(ct & 0xffffu), &steps))
              emit_hit(a, qid, opos, cpos - a.q_offsets[qid]);
            n_steps += steps;
          }
        }
      }
    }
  }
  __syncwarp();
  add_counter(&a.ctr[0], n_dist);
  add_counter(&a.ctr[1], n_seed);
  add_counter(&a.ctr[2], n_steps);
}

// first hit index of every query (hits sorted by packed key)
__global__ void hit_segments_kernel(const uint64_t *hits, uint64_t n, uint32_t nq, int shift,
                                    uint64_t *begin, const uint64_t *n_dev) {
  if (n_dev) n = *n_dev;
  for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi <= nq;
       qi += gridDim.x * blockDim.x) {
    const uint64_t key = (uint64_t)qi << shift;
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (hits[mid] < key)
        lo = mid + 1;
      else
        hi = mid;
    }
    begin[qi] = lo;
  }
}

// Chain filter (ChainFilter::Filter, src/chain_filter.cpp), one warp per
// query, over its hits in (database, query) position order; survivors are
// compacted to the front of the query's segment.  A hit only reads and
// writes its diagonal slot (diagonal % query length), so hits of different
// slots are independent and only a slot's own hits must be taken in order.
// The warp takes 32 hits at a time, one per lane, groups the lanes by slot
// (match.any) and runs rounds: in round r every lane whose hit is the r-th
// of its slot group applies it, so a round never touches a slot twice and
// a slot sees its hits in order.  The lanes' keep flags, in hit order, then
// place the survivors.  A query's (diagonal, end) slots live in the block's
// shared memory when its length fits `smem_slots` (one warp per block),
// else in `slots` (per-query scratch of query_length pairs).
constexpr int kChainSmemSlots = 4096;

__global__ void __launch_bounds__(32)
chain_kernel(DevParams p, const uint8_t *__restrict__ q, const uint8_t *__restrict__ db,
             const uint32_t *q_offsets, const uint32_t *q_lengths, const int32_t *cutoffs,
             const int32_t *matrix32, uint32_t nq, uint64_t *hits, const uint64_t *begin,
             int qbits, int dbits, uint2 *slots, uint32_t *kept_count, uint32_t smem_slots) {
  __shared__ __align__(16) int32_t tbl32[kWalkTableBytes / 4];
  extern __shared__ uint2 chain_slots[];
  load_walk_table(tbl32, matrix32, p.delimiter);
  __syncthreads();
  const char *tbl = reinterpret_cast<const char *>(tbl32);
  const uint64_t qmask = (1ull << qbits) - 1, dmask = (1ull << dbits) - 1;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1;
  for (uint32_t qi = blockIdx.x; qi < nq; qi += gridDim.x) {
    const uint64_t b = begin[qi], e = begin[qi + 1];
    if (b == e) {
      if (lane == 0) kept_count[qi] = 0;
      continue;
    }
    const uint8_t *qs = q + q_offsets[qi];
    const uint32_t qlen = q_lengths[qi];
    uint2 *slot = qlen <= smem_slots ? chain_slots : slots + q_offsets[qi] + qi;
    for (uint32_t i = lane; i < qlen; i += 32) slot[i] = make_uint2(0, 0);
    __syncwarp();
    const int cutoff = cutoffs[qi];
    uint64_t w = b;
    for (uint64_t i0 = b; i0 < e; i0 += 32) {
      // these 32 hits, one per lane (the compaction below only writes
      // positions before i0 + 32)
      const bool valid = i0 + lane < e;
      const uint64_t key = valid ? hits[i0 + lane] : 0;
      const uint32_t hq = (uint32_t)(key & qmask);
      const uint32_t hd = (uint32_t)((key >> qbits) & dmask);
      const uint32_t diagonal = qlen - 1 + hd - hq;
      const uint32_t si = valid ? diagonal % qlen : 0;
      // slot groups (an idle lane is a group of its own)
      const unsigned grp = __match_any_sync(0xffffffffu, valid ? si : (0x80000000u | lane));
      const int rank = __popc(grp & below);
      const int rounds = (int)__reduce_max_sync(0xffffffffu, (unsigned)__popc(grp));
      bool keep = false;
      for (int r = 0; r < rounds; ++r) {
        if (valid && rank == r) {
          uint2 sl = slot[si];  // x = diagonal, y = query end
          bool connected = false;
          if (sl.x == diagonal) {
            if (hq <= sl.y + 1) {
              connected = true;
            } else {
              // back-extension toward the chain end (ChainFilter::Connected):
              // the hq - 1 - end pairs before the hit
              connected = walk_reaches<-1>(qs + hq - 1, db + hd - 1, tbl, cutoff,
                                           hq - 1 - sl.y);
            }
          }
          sl.y = hq;
          if (!connected) sl.x = diagonal;
          slot[si] = sl;
          keep = !connected;
        }
        __syncwarp();  // the round's slot writes before the next round reads
      }
      const unsigned kept = __ballot_sync(0xffffffffu, keep);
      if (keep) hits[w + __popc(kept & below)] = key;
      w += __popc(kept);
    }
    if (lane == 0) kept_count[qi] = (uint32_t)(w - b);
    __syncwarp();
  }
}

// extension seeds: reverse at (q-1, d-1), forward at (q, d), absolute
// concatenated query / chunk positions
__device__ __forceinline__ uint32_t subject_of(const uint32_t *off, uint32_t nseq,
                                               uint32_t db_len, uint32_t pos);

// Extension list of the chained hits: one warp per query, lanes over its
// For every position p of a query in the concatenated buffer: the nearest
// delimiter at or before p (prev) and at or after p (next), within the
// query (its first and last codes are delimiters).  One warp per query,
// 32 positions per step with a running maximum (minimum) carried across
// steps.  The gapped DP cannot cross a delimiter, so these bound how far an
// extension can run along the query: for a protein query that is its end,
// for a translated query the end of the hit's frame.
__global__ void delim_dist_kernel(const uint8_t *q, const uint32_t *offsets,
                                  const uint32_t *lengths, uint32_t nq, int delim, uint32_t *prev,
                                  uint32_t *next) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t qi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; qi < nq; qi += warps) {
    const uint32_t off = offsets[qi], len = lengths[qi];
    uint32_t carry = off;  // the leading delimiter
    for (uint32_t b = 0; b < len; b += 32) {
      const uint32_t p = off + b + lane;
      uint32_t v = (b + lane < len && q[p] == delim) ? p : 0;
      v = max(v, carry);
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = max(v, u);
      }
      if (b + lane < len) prev[p] = v;
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
    carry = off + len - 1;  // the closing delimiter
    for (uint32_t b = 0; b < len; b += 32) {
      const uint32_t i = len - 1 - b - lane;  // positions from the end
      const uint32_t p = off + i;
      uint32_t v = (b + lane < len && q[p] == delim) ? p : 0xFFFFFFFFu;
      v = min(v, carry);
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = min(v, u);
      }
      if (b + lane < len) next[p] = v;
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

// kept hits (database order).  Reverse extension of hit h at h, forward at
// n_surv + h; neighbours[h] counts the query's kept hits within 256
// database residues of h (a cost-model feature).
__global__ void build_ext_kernel(const uint64_t *hits, const uint64_t *begin,
                                 const uint32_t *kept, const uint64_t *surv_off, uint32_t nq,
                                 const uint32_t *q_offsets, const uint32_t *q_lengths,
                                 const uint32_t *db_offsets, uint32_t nseq, uint32_t db_len,
                                 int qbits, int dbits, uint64_t n_surv, uint32_t *eq,
                                 uint32_t *ed, uint8_t *dir, uint32_t *elen0,
                                 uint32_t *elen1, uint32_t *eqid, uint32_t *neighbours,
                                 const uint64_t *n_dev, const uint32_t *qprev,
                                 const uint32_t *qnext, int features) {
  if (n_dev) n_surv = *n_dev;
  const uint64_t qmask = (1ull << qbits) - 1, dmask = (1ull << dbits) - 1;
  constexpr uint32_t kReach = 256;  // database residues either side
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t qi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; qi < nq; qi += warps) {
    const uint64_t b = begin[qi], o = surv_off[qi];
    const uint32_t qlen = q_lengths[qi];
    const uint32_t qoff = q_offsets[qi];
    const uint32_t nk = kept[qi];
    const uint64_t *kh = hits + b;
    for (uint32_t k = lane; k < nk; k += 32) {
      const uint64_t key = kh[k];
      const uint32_t hq = (uint32_t)(key & qmask);
      const uint32_t hd = (uint32_t)((key >> qbits) & dmask);
      if (neighbours) {
        // first kept hit at >= hd - kReach and first beyond hd + kReach
        const uint32_t lo_d = hd > kReach ? hd - kReach : 0, hi_d = hd + kReach;
        uint32_t lo = 0, hi = k;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if ((uint32_t)((kh[mid] >> qbits) & dmask) < lo_d) lo = mid + 1; else hi = mid;
        }
        const uint32_t first = lo;
        lo = k + 1;
        hi = nk;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if ((uint32_t)((kh[mid] >> qbits) & dmask) <= hi_d) lo = mid + 1; else hi = mid;
        }
        neighbours[o + k] = lo - first;
      }
      eq[o + k] = qoff + hq - 1;
      ed[o + k] = hd - 1;
      dir[o + k] = 1;
      eq[n_surv + o + k] = qoff + hq;
      ed[n_surv + o + k] = hd;
      dir[n_surv + o + k] = 0;
      if (features) {  // the cost model's inputs (remaining lengths, query)
        const uint32_t sj = subject_of(db_offsets, nseq, db_len, hd);
        const uint32_t s0 = db_offsets[sj], s1 = db_offsets[sj + 1] - 1;  // residues [s0, s1)
        elen0[o + k] = qprev ? (qoff + hq - 1) - qprev[qoff + hq - 1] : hq - 1;
        elen1[o + k] = hd - s0;
        eqid[o + k] = qi;
        elen0[n_surv + o + k] = qnext ? qnext[qoff + hq] - (qoff + hq) : qlen - 1 - hq;
        elen1[n_surv + o + k] = s1 - hd;
        eqid[n_surv + o + k] = qi;
      }
    }
  }
}

// Cost-model features of both extensions of every chained hit (one thread
// per hit: reverse extension h, forward extension n_surv + h).
__global__ void ext_features_kernel(const uint8_t *__restrict__ q, const uint8_t *__restrict__ db,
                                    int delim, const int32_t *__restrict__ matrix32,
                                    const int32_t *__restrict__ cutoffs, uint64_t n_surv,
                                    const uint32_t *eq, const uint32_t *ed,
                                    const uint32_t *elen0, const uint32_t *elen1,
                                    const uint32_t *eqid, const uint32_t *neighbours,
                                    float *feat, const uint64_t *n_dev) {
  if (n_dev) n_surv = *n_dev;
  for (uint64_t h = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; h < n_surv;
       h += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = h, f = n_surv + h;
    const int cutoff = cutoffs[eqid[h]];
    int best_r, steps_r, best_f, steps_f;
    diagonal_walk(q + eq[r], db + ed[r], -1, delim, matrix32, cutoff, &best_r, &steps_r);
    diagonal_walk(q + eq[f], db + ed[f], 1, delim, matrix32, cutoff, &best_f, &steps_f);
    float x[kFeat];
    extension_features(best_r, best_r + best_f, steps_r, elen0[r], elen1[r], true,
                       neighbours[h], x);
    for (int k = 0; k < kFeat; ++k) feat[r * kFeat + k] = x[k];
    extension_features(best_f, best_r + best_f, steps_f, elen0[f], elen1[f], false,
                       neighbours[h], x);
    for (int k = 0; k < kFeat; ++k) feat[f * kFeat + k] = x[k];
  }
}

// sort key: larger predicted cost first; ties keep extension order (the
// sort is stable and reads the low 16 bits)
// With n_dev the count is read on the device and entries n .. cap get the
// largest key (they sort last).
__global__ void cost_keys_kernel(const float *pred, const uint32_t *true_cells, uint64_t n,
                                 uint32_t *keys, uint32_t *vals, const uint64_t *n_dev,
                                 uint64_t cap) {
  if (n_dev) {
    const uint64_t m = *n_dev;
    for (uint64_t i = m + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap;
         i += (uint64_t)gridDim.x * blockDim.x) {
      keys[i] = 0xFFFFFFFFu;
      vals[i] = (uint32_t)i;
    }
    n = m;
  }
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float c = pred ? pred[i] : log2f(1.0f + (float)true_cells[i]);
    if (!(c > -64.0f)) c = -64.0f;
    if (c > 64.0f) c = 64.0f;
    // 16-bit keys (1/512 of a log2 unit): the order sort takes two passes
    const uint32_t u = min((uint32_t)((c + 64.0f) * 512.0f), 0xFFFFu);
    keys[i] = 0xFFFFu - u;
    vals[i] = (uint32_t)i;
  }
}

// appends (features, log2(1+cells)) of completed extensions to the log
__global__ void log_pairs_kernel(const float *feat, const uint32_t *cells_out, uint64_t n,
                                 float *log_x, float *log_y, unsigned long long *log_count,
                                 unsigned long long cap) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = cells_out[i];
    if (c == 0xFFFFFFFFu) continue;
    const unsigned long long slot = atomicAdd(log_count, 1ull);
    if (slot >= cap) continue;
    for (int k = 0; k < kFeat; ++k) log_x[slot * kFeat + k] = feat[i * kFeat + k];
    log_y[slot] = log2f(1.0f + (float)c);
  }
}

// sum |pred - log2(1+cells)| and count over completed extensions
__global__ void abs_error_kernel(const float *pred, const uint32_t *cells_out, uint64_t n,
                                 double *acc) {
  double s = 0.0, c = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t t = cells_out[i];
    if (t == 0xFFFFFFFFu) continue;
    s += fabs((double)pred[i] - (double)log2f(1.0f + (float)t));
    c += 1.0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc[0], s);
    atomicAdd(&acc[1], c);
  }
}

// ---- top-b merge -----------------------------------------------------------
__device__ __forceinline__ int alignment_comp(const gzb_result &a, const gzb_result &b) {
  if (a.score > b.score) return 1;
  if (a.score < b.score) return -1;
  const uint32_t aq = a.end_q - a.start_q, bq = b.end_q - b.start_q;
  if (aq > bq) return 1;
  if (aq < bq) return -1;
  const uint32_t as = a.end_d - a.start_d, bs = b.end_d - b.start_d;
  if (as > bs) return 1;
  if (as < bs) return -1;
  return (a.start_d < b.start_d) ? 1 : -1;
}

__device__ __forceinline__ bool is_contained(const gzb_result &a, const gzb_result &b) {
  return (a.start_q == b.start_q && a.start_d == b.start_d) ||
         (a.end_q == b.end_q && a.end_d == b.end_d) ||
         (a.start_q <= b.start_q && b.end_q <= a.end_q && a.start_d <= b.start_d &&
          b.end_d <= a.end_d);
}

__device__ __forceinline__ uint32_t subject_of(const uint32_t *off, uint32_t nseq,
                                               uint32_t db_len, uint32_t pos) {
  if (off[nseq - 1] <= pos && pos < db_len) return nseq - 1;
  uint32_t lo = 0, hi = nseq;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= pos)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo == 0 ? 0xFFFFFFFFu : lo - 1;
}


// Sort key of a candidate in AlignerCommon::AddResults' order (its stable
// sort by AlignmentComp): score, then query extent, then database extent
// descending, then database start ascending (k1 = score | query extent,
// k2 = database extent | ~database start, compared as unsigned).
// AlignmentComp is antisymmetric except on full ties, where it returns -1
// both ways and the reference's stable_sort keeps input order; equal keys
// are ordered by index here.
__device__ __forceinline__ ulonglong2 merge_key(const gzb_result &r) {
  return make_ulonglong2(
      ((unsigned long long)((uint32_t)r.score ^ 0x80000000u) << 32) |
          (uint32_t)(r.end_q - r.start_q),
      ((unsigned long long)(uint32_t)(r.end_d - r.start_d) << 32) | (uint32_t)~r.start_d);
}

__device__ __forceinline__ bool key_before(unsigned long long a1, unsigned long long a2,
                                           uint32_t ai, unsigned long long b1,
                                           unsigned long long b2, uint32_t bi) {
  return a1 > b1 || (a1 == b1 && (a2 > b2 || (a2 == b2 && ai < bi)));
}

// A lane's candidates as a binary heap of indices, first in `key_before`
// order at the root; element t at heap[32 t] (heap is offset by the lane).
// Sifts element t down through the m elements.
__device__ __forceinline__ void heap_sift(uint32_t *heap, const ulonglong2 *keys, uint32_t m,
                                          uint32_t t) {
  const uint32_t x = heap[32 * t];
  const ulonglong2 kx = keys[x];
  for (;;) {
    uint32_t c = 2 * t + 1;
    if (c >= m) break;
    uint32_t y = heap[32 * c];
    ulonglong2 ky = keys[y];
    if (c + 1 < m) {
      const uint32_t z = heap[32 * (c + 1)];
      const ulonglong2 kz = keys[z];
      if (key_before(kz.x, kz.y, z, ky.x, ky.y, y)) {
        c = c + 1;
        y = z;
        ky = kz;
      }
    }
    if (!key_before(ky.x, ky.y, y, kx.x, kx.y, x)) break;
    heap[32 * t] = y;
    t = c;
  }
  heap[32 * t] = x;
}

// One warp per query: the lanes build the candidates of the query's
// survivors, each lane keeps its own (i = lane, lane + 32, ...) as a heap in
// AlignerCommon::AddResults order, and the warp finds the next candidate as
// the best of the 32 heap roots; lane 0 merges it with the query's running
// top-b list, exactly as AddResults orders and prunes
// (src/aligner_common.h:147-274).
__global__ void merge_kernel(uint32_t nq, const uint64_t *hits, const uint64_t *begin,
                             const uint32_t *kept, const uint64_t *surv_off,
                             uint64_t n_surv, const uint32_t *eq, const uint32_t *ed,
                             const int32_t *escore, const uint32_t *q_offsets, int qbits,
                             int dbits, const uint32_t *db_offsets, uint32_t nseq,
                             uint32_t db_len, int32_t chunk_id, int max_results,
                             int max_one_subject, ulonglong2 *keys_all, uint32_t *heap_all,
                             gzb_result *results, uint32_t *counts, const uint64_t *n_dev,
                             const uint32_t *skip) {
  // a run whose buffers overflowed merges nothing (it is redone)
  if (skip && *skip) return;
  if (n_dev) n_surv = *n_dev;
  const uint64_t qmask = (1ull << qbits) - 1, dmask = (1ull << dbits) - 1;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  for (uint32_t qi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; qi < nq; qi += warps) {
    const uint32_t k = kept[qi];
    if (k == 0) continue;
    const uint64_t b = begin[qi], o = surv_off[qi];
    const uint32_t qoff = q_offsets[qi];
    ulonglong2 *keys = keys_all + o;
    uint32_t *heap = heap_all + o + lane;
    // candidate i of the query from its hit and its two extensions
    auto candidate = [&](uint32_t i) {
      const uint64_t key = hits[b + i];
      gzb_result r;
      r.chunk_id = chunk_id;
      r.subject_id = 0;
      r.hit_q = (uint32_t)(key & qmask);
      r.hit_d = (uint32_t)((key >> qbits) & dmask);
      r.score = escore[o + i] + escore[n_surv + o + i];
      r.start_q = eq[o + i] - qoff;
      r.start_d = ed[o + i];
      r.end_q = eq[n_surv + o + i] - qoff;
      r.end_d = ed[n_surv + o + i];
      return r;
    };
    uint32_t m = 0;
    for (uint32_t i = lane; i < k; i += 32) {
      keys[i] = merge_key(candidate(i));
      heap[32 * m] = i;
      ++m;
    }
    for (uint32_t t = m / 2; t-- > 0;) heap_sift(heap, keys, m, t);
    __syncwarp();
    uint32_t mine = m ? heap[0] : kNone;
    ulonglong2 mk = m ? keys[mine] : make_ulonglong2(0, 0);
    // lane 0's merge state: previous list of this query (earlier chunks)
    gzb_result *prev = results + (uint64_t)qi * max_results;
    const uint32_t n_prev = counts[qi];
    gzb_result old[32];
    const uint32_t n_old = n_prev < 32 ? n_prev : 32;
    if (lane == 0)
      for (uint32_t i = 0; i < n_old; ++i) old[i] = prev[i];
    uint32_t ri = 0, n_out = 0, left = k;
    // per-subject start lists of this chunk (subject, size, entries)
    uint32_t subj[32];
    uint32_t subj_n[32];
    uint32_t sp_pos[32][4];
    uint32_t sp_id[32][4];
    uint32_t n_subj = 0;
    for (;;) {
      // first untaken candidate of the warp: the best of the lanes' roots
      uint32_t g = mine;
      unsigned long long g1 = mk.x, g2 = mk.y;
      for (int d = 16; d >= 1; d >>= 1) {
        const uint32_t og = __shfl_xor_sync(0xffffffffu, g, d);
        const unsigned long long o1 = __shfl_xor_sync(0xffffffffu, g1, d);
        const unsigned long long o2 = __shfl_xor_sync(0xffffffffu, g2, d);
        if (og != kNone && (g == kNone || key_before(o1, o2, og, g1, g2, g))) {
          g = og;
          g1 = o1;
          g2 = o2;
        }
      }
      int popped = -1, cont = 0;
      if (lane == 0) {
        if ((int)n_out < max_results && (left > 0 || ri < n_old)) {
          cont = 1;
          gzb_result a;
          const gzb_result cand = left ? candidate(g) : gzb_result{};
          bool take_added;
          if (left == 0)
            take_added = false;
          else if (ri == n_old)
            take_added = true;
          else
            take_added = alignment_comp(old[ri], cand) < 0;
          if (take_added) {
            a = cand;
            a.subject_id = (int32_t)subject_of(db_offsets, nseq, db_len, a.start_d);
            popped = (int)g;
            --left;
          } else {
            a = old[ri++];
          }
          bool keep = true;
          if (a.chunk_id == chunk_id) {
            keep = false;
            uint32_t si = 0;
            while (si < n_subj && subj[si] != (uint32_t)a.subject_id) ++si;
            bool room = true;
            if (si == n_subj) {
              if (n_subj == 32) {
                room = false;  // cannot exceed max_results subjects
              } else {
                subj[si] = (uint32_t)a.subject_id;
                subj_n[si] = 0;
                ++n_subj;
              }
            }
            const uint32_t cnt = room ? subj_n[si] : 0;
            if (room && (int)cnt < max_one_subject && cnt < 4) {
              // std::lower_bound on .position, step for step
              uint32_t first = 0, len = cnt;
              while (len > 0) {
                const uint32_t half = len / 2, mid = first + half;
                if (sp_pos[si][mid] < a.start_d) {
                  first = mid + 1;
                  len = len - half - 1;
                } else {
                  len = half;
                }
              }
              const uint32_t ins = first;
              uint32_t it = first;
              len = cnt - first;
              uint32_t f2 = first;
              while (len > 0) {
                const uint32_t half = len / 2, mid = f2 + half;
                if (sp_pos[si][mid] < a.end_d) {
                  f2 = mid + 1;
                  len = len - half - 1;
                } else {
                  len = half;
                }
              }
              bool ok = true;
              for (; it != f2; ++it) {
                if (is_contained(prev[sp_id[si][it]], a)) {
                  ok = false;
                  break;
                }
              }
              if (ok) {
                for (uint32_t t = cnt; t > ins; --t) {
                  sp_pos[si][t] = sp_pos[si][t - 1];
                  sp_id[si][t] = sp_id[si][t - 1];
                }
                sp_pos[si][ins] = a.start_q;
                sp_id[si][ins] = n_out;
                subj_n[si] = cnt + 1;
                keep = true;
              }
            }
          }
          if (keep) prev[n_out++] = a;
        }
      }
      cont = __shfl_sync(0xffffffffu, cont, 0);
      if (!cont) break;
      popped = __shfl_sync(0xffffffffu, popped, 0);
      if (popped >= 0 && (uint32_t)popped % 32 == (uint32_t)lane) {
        // the candidate taken is this lane's root
        --m;
        if (m) {
          heap[0] = heap[32 * m];
          heap_sift(heap, keys, m, 0);
          mine = heap[0];
          mk = keys[mine];
        } else {
          mine = kNone;
        }
      }
      __syncwarp();
    }
    if (lane == 0) counts[qi] = n_out;
  }
}

}  // namespace gzb

using namespace gzb;

// ===========================================================================
struct gzb_engine {
  int device = 0;
  gzb_params params{};
  DevParams dp{};
  bool have_params = false;
  DBuf matrix32;
  // database
  int32_t chunk_id = 0;
  DBuf db_buf;
  uint64_t db_len = 0;
  DBuf db_offsets;
  uint32_t nseq = 0;
  DevIndex X;
  std::vector<DBuf> index_bufs;
  bool have_db = false;
  // queries
  DBuf q_buf, q_offsets, q_lengths, q_cut, q_trig;
  DBuf q_off64, q_prep;  // query preparation on the device: 64-bit offsets, scratch
  DBuf q_prev, q_next;  // nearest delimiters of every query position
  uint64_t q_len = 0;
  uint32_t nq = 0;
  uint32_t max_qlen = 0;
  DevLists L;
  std::vector<DBuf> list_bufs;
  bool have_queries = false;
  // results
  DBuf results, counts;
  // scratch
  DBuf tmp, hits, hits_alt, mwork, mwork_alt, begin, kept, surv_off, slots, eq, ed, edir,
      escore, heap, ctr, misc, hits_copy;
  int qbits = 1, dbits = 1;
  // schedule of the gapped stage
  DBuf elen0, elen1, eqid, efeat, epred, ecells, okeys, okeys2, oidx, oidx2, queue, prev_cells,
      model_d, mae_acc, log_x, log_y, log_ctr;
  uint64_t prev_cells_n = 0;
  DBuf codeflag;
  uint64_t db_check = 0;     // of the resident chunk (index cache key)
  // build results step
  DBuf tb_redo;
  DBuf tb_cols, tb_band_off, tb_band, tb_ops_bytes, tb_ops_off, tb_rows, tb_rows_off, tb_ops,
      tb_row_meta, tb_score, tb_p0, tb_p1, tb_out, tb_stats, tb_scratch;
  uint64_t pred_n = 0;       // extensions with a prediction in epred (last run)
  DBuf enb;                  // per surviving hit: chained neighbours (cost feature)
  int tile[3][kTileParameters] = {
      {-1, -1, -1, -1, -1}, {-1, -1, -1, -1, -1}, {-1, -1, -1, -1, -1}};
  // [schedule][which], -1 = default
  bool logging = false;
  uint64_t log_cap = 0;
  bool have_model = false;
  float last_mae = -1.0f;
  uint64_t last_mae_n = 0;
  uint32_t *spill = nullptr;
  size_t spill_cap = 0;
  uint32_t *gcounters = nullptr;
  unsigned long long *gcells = nullptr;
  int2 *band_pool = nullptr;
  int band_wmask = 0;
  uint64_t hit_cap = 1ull << 22, mwork_cap = 1ull << 22;
  gzb_counters counters{};
  float stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
  cudaEvent_t ev[7] = {};
  // stored database chunks (gzb_engine_swap_database): each holds a chunk's
  // codes, offsets and the ten index arrays, compact
  struct DbSlot {
    bool have = false;
    bool pending = false;          // a prefetch's copies may still run
    int32_t chunk_id = 0;
    DBuf db_buf, db_offsets, codeflag;
    DBuf arrays[10];
    uint64_t db_len = 0, db_check = 0;
    uint32_t nseq = 0;
    DevIndex X;
    cudaEvent_t ready = nullptr;   // recorded after a prefetch's copies
  };
  std::vector<DbSlot> db_slots;
  bool x_in_arrays = false;        // X points into index_bufs[40..49]
  // graph mode: captured presearch graphs, keyed by what they depend on
  struct GraphEntry {
    uint64_t key;
    cudaGraphExec_t exec;
    uint64_t launches;             // kernels in the graph
    uint64_t used;                 // last use (for eviction)
  };
  bool graph = false;
  std::vector<GraphEntry> graphs;
  cudaStream_t gstream = nullptr;
  cudaEvent_t gev_in = nullptr, gev_out = nullptr;
  DBuf plan;                       // device counts and the report
  uint64_t *report_h = nullptr;    // pinned copy of the report
  uint64_t graph_captures = 0, graph_replays = 0, graph_fallbacks = 0, graph_clock = 0;
};

namespace {

int bits_for(uint64_t v) {  // bits to hold values in [0, v]
  int b = 1;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

// CUB wrappers using the engine's growable temp buffer
int sort_keys_u64(gzb_engine *e, uint64_t *keys, uint64_t *alt, uint64_t n, int end_bit,
                  cudaStream_t s, uint64_t **result) {
  cub::DoubleBuffer<uint64_t> db(keys, alt);
  size_t tb = 0;
  GZB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int64_t)n, 0, end_bit, s));
  GZB_TRY(e->tmp.ensure(tb));
  GZB_CUDA(cub::DeviceRadixSort::SortKeys(e->tmp.p, tb, db, (int64_t)n, 0, end_bit, s));
  *result = db.Current();
  return GZB_OK;
}

int select_flagged_index(gzb_engine *e, const uint8_t *flags, uint64_t n, uint32_t *out,
                         uint64_t *n_out, cudaStream_t s) {
  // indices i with flags[i] != 0, in order
  GZB_TRY(e->misc.ensure(8));
  thrust::counting_iterator<uint32_t> it(0);
  size_t tb = 0;
  GZB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, flags, out, e->misc.as<uint64_t>(),
                                      (int64_t)n, s));
  GZB_TRY(e->tmp.ensure(tb));
  GZB_CUDA(cub::DeviceSelect::Flagged(e->tmp.p, tb, it, flags, out, e->misc.as<uint64_t>(),
                                      (int64_t)n, s));
  uint64_t cnt = 0;
  GZB_CUDA(cudaMemcpyAsync(&cnt, e->misc.p, 8, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  *n_out = cnt;
  return GZB_OK;
}

template <class T>
int select_flagged(gzb_engine *e, const T *in, const uint8_t *flags, uint64_t n, T *out,
                   uint64_t *n_out, cudaStream_t s) {
  GZB_TRY(e->misc.ensure(8));
  size_t tb = 0;
  GZB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, in, flags, out, e->misc.as<uint64_t>(),
                                      (int64_t)n, s));
  GZB_TRY(e->tmp.ensure(tb));
  GZB_CUDA(cub::DeviceSelect::Flagged(e->tmp.p, tb, in, flags, out, e->misc.as<uint64_t>(),
                                      (int64_t)n, s));
  uint64_t cnt = 0;
  GZB_CUDA(cudaMemcpyAsync(&cnt, e->misc.p, 8, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  *n_out = cnt;
  return GZB_OK;
}

template <class TIn, class TOut>
int exclusive_sum(gzb_engine *e, const TIn *in, TOut *out, uint64_t n, cudaStream_t s) {
  size_t tb = 0;
  GZB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int64_t)n, s));
  GZB_TRY(e->tmp.ensure(tb));
  GZB_CUDA(cub::DeviceScan::ExclusiveSum(e->tmp.p, tb, in, out, (int64_t)n, s));
  return GZB_OK;
}

// sets *bad when a byte of p[0, n) is 32 or more (p 16-byte aligned)
__global__ void code_range_kernel(const uint8_t *p, uint64_t n, unsigned int *bad) {
  const uint64_t n16 = n / 16;
  const uint4 *p4 = reinterpret_cast<const uint4 *>(p);
  uint32_t acc = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 v = p4[i];
    acc |= v.x | v.y | v.z | v.w;
  }
  if (blockIdx.x == 0 && threadIdx.x < 16 && n16 * 16 + threadIdx.x < n)
    acc |= p[n16 * 16 + threadIdx.x];
  if (acc & 0xE0E0E0E0u) atomicOr(bad, 1u);
}

// the query cutoffs the engine takes (1..32767) and triggers (int16)
__global__ void cutoff_range_kernel(const int32_t *cut, const int32_t *trig, uint32_t n,
                                    unsigned int *bad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (cut[i] < 1 || cut[i] > 32767 || trig[i] < -32768 || trig[i] > 32767) atomicOr(bad, 1u);
}

// cut[idx[i]] = c[i], trig[idx[i]] = t[i]
__global__ void scatter_cutoffs_kernel(const uint32_t *idx, const int32_t *c, const int32_t *t,
                                       uint32_t n, int32_t *cut, int32_t *trig) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    cut[idx[i]] = c[i];
    trig[idx[i]] = t[i];
  }
}

// Uploads `len` residue codes between kPad delimiter bytes on each side and
// checks that every code is below 32 (the kernels' score tables are 32
// wide).  Synchronises `s`.
int upload_padded(DBuf &buf, DBuf &flag, const uint8_t *codes, uint64_t len, uint8_t delim,
                  cudaStream_t s) {
  GZB_TRY(buf.ensure(len + 2 * kPad));
  GZB_TRY(flag.ensure(4));
  GZB_CUDA(cudaMemsetAsync(buf.p, delim, len + 2 * kPad, s));
  GZB_CUDA(cudaMemcpyAsync((uint8_t *)buf.p + kPad, codes, len, cudaMemcpyHostToDevice, s));
  GZB_CUDA(cudaMemsetAsync(flag.p, 0, 4, s));
  code_range_kernel<<<grid1(len / 16 + 1, 256), 256, 0, s>>>((const uint8_t *)buf.p + kPad, len,
                                                               flag.as<unsigned int>());
  GZB_CUDA(cudaGetLastError());
  unsigned int bad = 0;
  GZB_CUDA(cudaMemcpyAsync(&bad, flag.p, 4, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  GZB_CHECK(bad == 0, GZB_ERR_INVALID, "residue codes must be below 32");
  return GZB_OK;
}

template <class T>
int upload(DBuf &buf, const T *h, uint64_t n, cudaStream_t s) {
  GZB_TRY(buf.ensure(sizeof(T) * (n ? n : 1)));
  if (n) GZB_CUDA(cudaMemcpyAsync(buf.p, h, sizeof(T) * n, cudaMemcpyHostToDevice, s));
  return GZB_OK;
}

int build_csr(gzb_engine *e, const uint64_t *pairs, uint64_t n, uint32_t **keys,
              uint32_t **offsets, uint32_t **values, uint64_t *nkeys, int slot,
              cudaStream_t s) {
  DBuf &flags = e->index_bufs[slot];
  DBuf &starts = e->index_bufs[slot + 1];
  DBuf &kbuf = e->index_bufs[slot + 2];
  DBuf &obuf = e->index_bufs[slot + 3];
  DBuf &vbuf = e->index_bufs[slot + 4];
  GZB_TRY(flags.ensure(n + 1));
  GZB_TRY(starts.ensure(4 * (n + 1)));
  if (n) {
    key_start_flags<<<grid1(n, 256), 256, 0, s>>>(pairs, n, flags.as<uint8_t>());
    GZB_CUDA(cudaGetLastError());
  }
  uint64_t nseg = 0;
  if (n) GZB_TRY(select_flagged_index(e, flags.as<uint8_t>(), n, starts.as<uint32_t>(), &nseg, s));
  GZB_TRY(kbuf.ensure(4 * (nseg + 1)));
  GZB_TRY(obuf.ensure(4 * (nseg + 1)));
  GZB_TRY(vbuf.ensure(4 * (n + 1)));
  csr_fill<<<grid1(n + nseg + 1, 256), 256, 0, s>>>(pairs, n, starts.as<uint32_t>(), nseg,
                                                      kbuf.as<uint32_t>(), obuf.as<uint32_t>(),
                                                      vbuf.as<uint32_t>());
  GZB_CUDA(cudaGetLastError());
  *keys = kbuf.as<uint32_t>();
  *offsets = obuf.as<uint32_t>();
  *values = vbuf.as<uint32_t>();
  *nkeys = nseg;
  return GZB_OK;
}

int check_engine(gzb_engine *e) {
  GZB_CHECK(e, GZB_ERR_INVALID, "null engine");
  GZB_CUDA(cudaSetDevice(e->device));
  return GZB_OK;
}

}  // namespace

extern "C" int gzb_engine_create(int device, gzb_engine **out) {
  GZB_CHECK(out, GZB_ERR_INVALID, "null output handle");
  int ndev = 0;
  GZB_CUDA(cudaGetDeviceCount(&ndev));
  GZB_CHECK(device >= 0 && device < ndev, GZB_ERR_INVALID, "no CUDA device %d", device);
  GZB_CUDA(cudaSetDevice(device));
  gzb_engine *e = new (std::nothrow) gzb_engine();
  GZB_CHECK(e, GZB_ERR_NOMEM, "host allocation failed");
  e->device = device;
  e->index_bufs.resize(50);
  e->list_bufs.resize(20);
  cudaError_t err = cudaMalloc(&e->gcounters, 64);
  if (err == cudaSuccess) err = cudaMalloc(&e->gcells, 8);
  if (err == cudaSuccess) err = cudaMemset(e->gcounters, 0, 64);
  if (err == cudaSuccess) err = cudaMemset(e->gcells, 0, 8);
  for (int i = 0; i < 7 && err == cudaSuccess; ++i) err = cudaEventCreate(&e->ev[i]);
  if (err != cudaSuccess) {
    gzb_engine_destroy(e);
    return cuda_error(err, "engine set-up", __FILE__, __LINE__);
  }
  *out = e;
  return GZB_OK;
}

extern "C" int gzb_engine_destroy(gzb_engine *e) {
  if (!e) return GZB_OK;
  cudaSetDevice(e->device);
  for (auto &b : e->index_bufs) b.release();
  for (auto &b : e->list_bufs) b.release();
  DBuf *all[] = {&e->matrix32, &e->db_buf, &e->db_offsets, &e->q_buf, &e->q_offsets,
                 &e->q_prev, &e->q_next, &e->q_off64, &e->q_prep,
                 &e->q_lengths, &e->q_cut, &e->q_trig, &e->results, &e->counts,
                 &e->tmp, &e->hits, &e->hits_alt, &e->mwork, &e->mwork_alt,
                 &e->begin, &e->kept, &e->surv_off, &e->slots, &e->eq, &e->ed, &e->edir,
                 &e->escore, &e->heap, &e->ctr, &e->misc,
                 &e->hits_copy, &e->elen0, &e->elen1, &e->eqid, &e->efeat, &e->epred,
                 &e->ecells, &e->okeys, &e->okeys2, &e->oidx, &e->oidx2, &e->queue,
                 &e->prev_cells, &e->model_d, &e->mae_acc, &e->log_x, &e->log_y,
                 &e->log_ctr, &e->enb, &e->codeflag, &e->tb_cols, &e->tb_band_off,
                 &e->tb_redo,
                 &e->tb_band, &e->tb_ops_bytes, &e->tb_ops_off, &e->tb_rows, &e->tb_rows_off,
                 &e->tb_ops, &e->tb_row_meta, &e->tb_score, &e->tb_p0, &e->tb_p1, &e->tb_out, &e->tb_stats,
                 &e->tb_scratch};
  for (DBuf *b : all) b->release();
  for (auto &g : e->graphs) cudaGraphExecDestroy(g.exec);
  e->graphs.clear();
  if (e->gstream) cudaStreamSynchronize(e->gstream);
  if (e->gstream) cudaStreamDestroy(e->gstream);
  if (e->gev_in) cudaEventDestroy(e->gev_in);
  if (e->gev_out) cudaEventDestroy(e->gev_out);
  if (e->report_h) cudaFreeHost(e->report_h);
  e->plan.release();
  for (auto &slot : e->db_slots) {
    if (slot.ready) cudaEventSynchronize(slot.ready);
    slot.db_buf.release();
    slot.db_offsets.release();
    slot.codeflag.release();
    for (auto &b : slot.arrays) b.release();
    if (slot.ready) cudaEventDestroy(slot.ready);
  }
  cudaFree(e->spill);
  cudaFree(e->gcounters);
  cudaFree(e->gcells);
  cudaFree(e->band_pool);
  for (int i = 0; i < 7; ++i)
    if (e->ev[i]) cudaEventDestroy(e->ev[i]);
  delete e;
  return GZB_OK;
}

extern "C" int gzb_engine_set_params(gzb_engine *e, const gzb_params *p) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(p, GZB_ERR_INVALID, "null params");
  GZB_CHECK(p->number_letters > 0 && p->number_letters < 32, GZB_ERR_INVALID,
            "number_letters out of range");
  GZB_CHECK(p->map_size > 0 && p->map_size <= 32, GZB_ERR_INVALID, "map_size out of range");
  GZB_CHECK(p->subsequence_length >= 1 && p->subsequence_length <= 16, GZB_ERR_INVALID,
            "subsequence_length must be 1..16");
  GZB_CHECK(p->max_hash_length >= 1 && p->max_hash_length <= 16, GZB_ERR_INVALID,
            "max_hash_length out of range");
  GZB_CHECK(p->max_number_results >= 1 && p->max_number_results <= 32, GZB_ERR_INVALID,
            "max_number_results must be 1..32");
  GZB_CHECK(p->max_number_one_subject_results >= 1, GZB_ERR_INVALID,
            "max_number_one_subject_results must be >= 1");
  GZB_CHECK(p->gap_open >= 0 && p->gap_extension >= 0, GZB_ERR_INVALID, "negative gap");
  GZB_CHECK(p->delimiter >= 0 && p->delimiter < 32, GZB_ERR_INVALID, "delimiter must be 0..31");
  for (int i = 0; i < p->number_letters * p->number_letters; ++i)
    GZB_CHECK(p->score_matrix[i] > -32768 && p->score_matrix[i] < 32768, GZB_ERR_INVALID,
              "score matrix entries must fit int16");
  e->params = *p;
  DevParams &d = e->dp;
  memset(&d, 0, sizeof(d));
  d.delimiter = p->delimiter;
  d.number_letters = p->number_letters;
  d.map_size = p->map_size;
  d.max_indexing_code = p->max_indexing_code;
  d.seed_threshold = p->seed_threshold;
  d.max_hash_length = p->max_hash_length;
  d.min_hash_length = p->min_hash_length;
  d.subsequence_length = p->subsequence_length;
  d.max_member_distance = p->max_member_distance;
  d.distance_threshold = p->distance_threshold;
  int shift = 0;
  for (uint32_t c = 1; c < (uint32_t)p->max_indexing_code + 1u; c <<= 1) ++shift;
  d.shift = shift;
  GZB_CHECK(shift * p->max_hash_length <= 32, GZB_ERR_INVALID, "hash does not fit 32 bits");
  for (int i = 0; i < 32; ++i) {
    const int r = p->hash_code_map[i];
    d.hash_map[i] = (i < p->map_size && r <= p->max_indexing_code) ? (uint8_t)(r + 1) : 0;
    d.sim_map[i] = p->similarity_code_map[i];
    GZB_CHECK(i >= p->map_size || p->similarity_code_map[i] < 16, GZB_ERR_INVALID,
              "similarity codes must be < 16");
  }
  for (int c = 0; c <= p->max_indexing_code && c < 31; ++c) d.code_scores[c + 1] = p->code_scores[c];
  // 32x32 score matrix tile (rows = database code)
  int32_t m[32 * 32];
  memset(m, 0, sizeof(m));
  for (int r = 0; r < p->number_letters; ++r)
    for (int c = 0; c < p->number_letters; ++c)
      m[r * 32 + c] = p->score_matrix[r * p->number_letters + c];
  GZB_TRY(e->matrix32.ensure(sizeof(m)));
  GZB_CUDA(cudaMemcpy(e->matrix32.p, m, sizeof(m), cudaMemcpyHostToDevice));
  e->have_params = true;
  return GZB_OK;
}

namespace {

// ---- device index cache ----------------------------------------------------
// (blob format: gzb_blob.h)

uint64_t index_fingerprint(const gzb_engine *e) { return params_fingerprint(e->params); }

IndexHeader header_of(const gzb_engine *e) {
  IndexHeader h;
  memset(&h, 0, sizeof(h));
  h.magic = kIndexMagic;
  h.fingerprint = index_fingerprint(e);
  h.db_len = e->db_len;
  h.nseq = e->nseq;
  h.db_check = e->db_check;
  h.n_nc_keys = e->X.n_nc_keys;
  h.n_nc_values = e->X.n_nc_values;
  h.n_rep_keys = e->X.params_clustering ? e->X.n_rep_keys : 0;
  h.n_reps = e->X.params_clustering ? e->X.n_reps : 0;
  h.n_members = e->X.params_clustering ? e->X.n_members : 0;
  return h;
}

}  // namespace

extern "C" int gzb_engine_set_database(gzb_engine *e, int32_t chunk_id, const uint8_t *codes,
                                       uint64_t length, const uint32_t *offsets,
                                       uint32_t number_sequences, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_params, GZB_ERR_INVALID, "set_params first");
  GZB_CHECK(codes && offsets && number_sequences > 0 && length > 0, GZB_ERR_INVALID,
            "empty database");
  GZB_CHECK(length < (1ull << 31), GZB_ERR_OVERFLOW,
            "database chunk of %llu residues exceeds 2^31", (unsigned long long)length);
  cudaStream_t s = (cudaStream_t)stream;
  e->have_db = false;
  e->x_in_arrays = false;
  e->chunk_id = chunk_id;
  e->db_len = length;
  e->nseq = number_sequences;
  e->db_check = db_check(codes, length, offsets, number_sequences);
  GZB_TRY(upload_padded(e->db_buf, e->codeflag, codes, length, (uint8_t)e->params.delimiter, s));
  GZB_TRY(upload(e->db_offsets, offsets, number_sequences + 1, s));
  const uint8_t *db = e->db_buf.as<uint8_t>() + kPad;
  std::vector<DBuf> &B = e->index_bufs;
  // 1. (hash, position) pairs
  DBuf &pairs = B[0], &pairs_alt = B[1];
  GZB_TRY(pairs.ensure(8 * (length + 1)));
  GZB_TRY(pairs_alt.ensure(8 * (length + 1)));
  GZB_TRY(e->ctr.ensure(64));
  GZB_CUDA(cudaMemsetAsync(e->ctr.p, 0, 64, s));
  db_pairs_kernel<<<grid1(length, 256, 148 * 64), 256, 0, s>>>(
      e->dp, db, length, pairs.as<uint64_t>(), e->ctr.as<unsigned long long>());
  GZB_CUDA(cudaGetLastError());
  uint64_t np = 0;
  GZB_CUDA(cudaMemcpyAsync(&np, e->ctr.p, 8, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  uint64_t *sorted = nullptr;
  GZB_TRY(sort_keys_u64(e, pairs.as<uint64_t>(), pairs_alt.as<uint64_t>(), np, 64, s, &sorted));
  uint64_t *other = sorted == pairs.as<uint64_t>() ? pairs_alt.as<uint64_t>() : pairs.as<uint64_t>();
  DevIndex &X = e->X;
  X = DevIndex();
  X.params_clustering = e->params.clustering != 0;
  if (!e->params.clustering) {
    GZB_TRY(build_csr(e, sorted, np, &X.nc_keys, &X.nc_offsets, &X.nc_values, &X.n_nc_keys, 10, s));
    X.n_nc_values = np;
    // empty representative / member indexes
    GZB_TRY(B[20].ensure(16));
    GZB_TRY(B[21].ensure(16));
    GZB_CUDA(cudaMemsetAsync(B[20].p, 0, 16, s));
    GZB_CUDA(cudaMemsetAsync(B[21].p, 0, 16, s));
    X.rep_keys = B[20].as<uint32_t>();
    X.rep_offsets = B[20].as<uint32_t>();
    X.rep_cluster_ids = B[20].as<uint32_t>();
    X.rep_positions = B[20].as<uint32_t>();
    X.member_offsets = B[21].as<uint32_t>();
    X.member_positions = B[21].as<uint32_t>();
    X.rep_windows = (uint64_t *)B[21].p;
    GZB_CUDA(cudaStreamSynchronize(s));
    e->have_db = true;
    return GZB_OK;
  }
  // 2. clustering
  DBuf &fstart = B[2], &state = B[3], &window = B[4], &bstart = B[5], &rep_of = B[6],
       &mcount = B[7], &is_nc = B[8], &is_rep = B[9];
  GZB_TRY(fstart.ensure(np + 1));
  GZB_TRY(state.ensure(np + 1));
  GZB_TRY(window.ensure(8 * (np + 1)));
  GZB_TRY(bstart.ensure(4 * (np + 1)));
  GZB_TRY(rep_of.ensure(4 * (np + 1)));
  GZB_TRY(mcount.ensure(4 * (np + 1)));
  GZB_TRY(is_nc.ensure(np + 1));
  GZB_TRY(is_rep.ensure(np + 1));
  DBuf &is_mem = B[30];
  GZB_TRY(is_mem.ensure(np + 1));
  db_entry_kernel<<<grid1(np, 256, 148 * 64), 256, 0, s>>>(
      e->dp, db, sorted, np, fstart.as<uint8_t>(), state.as<uint8_t>(), window.as<uint64_t>());
  GZB_CUDA(cudaGetLastError());
  uint64_t nb = 0;
  GZB_TRY(select_flagged_index(e, fstart.as<uint8_t>(), np, bstart.as<uint32_t>(), &nb, s));
  cluster_kernel<<<grid1(nb * 32, 256, 148 * 16), 256, 0, s>>>(
      bstart.as<uint32_t>(), nb, np, state.as<uint8_t>(), window.as<uint64_t>(),
      rep_of.as<uint32_t>(), e->params.max_member_distance);
  GZB_CUDA(cudaGetLastError());
  GZB_CUDA(cudaMemsetAsync(mcount.p, 0, 4 * (np + 1), s));
  member_count_kernel<<<grid1(np, 256), 256, 0, s>>>(state.as<uint8_t>(), rep_of.as<uint32_t>(),
                                                      np, mcount.as<uint32_t>());
  GZB_CUDA(cudaGetLastError());
  classify_kernel<<<grid1(np, 256), 256, 0, s>>>(state.as<uint8_t>(), mcount.as<uint32_t>(), np,
                                                  is_nc.as<uint8_t>(), is_rep.as<uint8_t>(),
                                                  is_mem.as<uint8_t>());
  GZB_CUDA(cudaGetLastError());
  // residual index
  uint64_t nnc = 0;
  GZB_TRY(select_flagged(e, sorted, is_nc.as<uint8_t>(), np, other, &nnc, s));
  GZB_TRY(build_csr(e, other, nnc, &X.nc_keys, &X.nc_offsets, &X.nc_values, &X.n_nc_keys, 10, s));
  X.n_nc_values = nnc;
  GZB_CUDA(cudaStreamSynchronize(s));
  // representatives (order kept: hash, then position)
  uint64_t nrep = 0;
  GZB_TRY(select_flagged(e, sorted, is_rep.as<uint8_t>(), np, other, &nrep, s));
  DBuf &rwin = B[32];
  GZB_TRY(rwin.ensure(8 * (nrep + 1)));
  uint64_t nrw = 0;
  GZB_TRY(select_flagged(e, window.as<uint64_t>(), is_rep.as<uint8_t>(), np,
                         rwin.as<uint64_t>(), &nrw, s));
  X.rep_windows = rwin.as<uint64_t>();
  uint32_t *rk, *ro, *rv;
  uint64_t nrk = 0;
  GZB_TRY(build_csr(e, other, nrep, &rk, &ro, &rv, &nrk, 15, s));
  X.rep_keys = rk;
  X.rep_offsets = ro;
  X.rep_positions = rv;
  X.n_rep_keys = nrk;
  X.n_reps = nrep;
  DBuf &rep_entries = B[22], &cid_of_entry = B[23], &cids = B[24];
  GZB_TRY(rep_entries.ensure(4 * (nrep + 1)));
  GZB_TRY(cid_of_entry.ensure(4 * (np + 1)));
  GZB_TRY(cids.ensure(4 * (nrep + 1)));
  uint64_t tmpn = 0;
  GZB_TRY(select_flagged_index(e, is_rep.as<uint8_t>(), np, rep_entries.as<uint32_t>(), &tmpn, s));
  scatter_cluster_ids<<<grid1(nrep, 256), 256, 0, s>>>(rep_entries.as<uint32_t>(), nrep,
                                                        cid_of_entry.as<uint32_t>(),
                                                        cids.as<uint32_t>());
  GZB_CUDA(cudaGetLastError());
  X.rep_cluster_ids = cids.as<uint32_t>();
  // members grouped by cluster, position order inside
  DBuf &mem_entries = B[25], &mpairs = B[26], &mpairs_alt = B[27], &mcnt = B[28],
       &moff = B[29], &mpos = B[31];
  GZB_TRY(mem_entries.ensure(4 * (np + 1)));
  uint64_t nm = 0;
  GZB_TRY(select_flagged_index(e, is_mem.as<uint8_t>(), np, mem_entries.as<uint32_t>(), &nm, s));
  GZB_TRY(mpairs.ensure(8 * (nm + 1)));
  GZB_TRY(mpairs_alt.ensure(8 * (nm + 1)));
  GZB_TRY(mcnt.ensure(4 * (nrep + 1)));
  GZB_TRY(moff.ensure(4 * (nrep + 2)));
  GZB_TRY(mpos.ensure(4 * (nm + 1)));
  GZB_CUDA(cudaMemsetAsync(mcnt.p, 0, 4 * (nrep + 1), s));
  member_pairs_kernel<<<grid1(nm, 256), 256, 0, s>>>(mem_entries.as<uint32_t>(), nm,
                                                      rep_of.as<uint32_t>(),
                                                      cid_of_entry.as<uint32_t>(), sorted,
                                                      mpairs.as<uint64_t>(), mcnt.as<uint32_t>());
  GZB_CUDA(cudaGetLastError());
  uint64_t *msorted = nullptr;
  GZB_TRY(sort_keys_u64(e, mpairs.as<uint64_t>(), mpairs_alt.as<uint64_t>(), nm, 64, s, &msorted));
  low32<<<grid1(nm, 256), 256, 0, s>>>(msorted, nm, mpos.as<uint32_t>());
  GZB_CUDA(cudaGetLastError());
  GZB_TRY(exclusive_sum(e, mcnt.as<uint32_t>(), moff.as<uint32_t>(), nrep + 1, s));
  X.member_offsets = moff.as<uint32_t>();
  X.member_positions = mpos.as<uint32_t>();
  X.n_members = nm;
  GZB_CUDA(cudaStreamSynchronize(s));
  e->have_db = true;
  return GZB_OK;
}

extern "C" int gzb_engine_index_bytes(gzb_engine *e, uint64_t *bytes) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(bytes, GZB_ERR_INVALID, "null argument");
  GZB_CHECK(e->have_db, GZB_ERR_INVALID, "no database chunk");
  *bytes = index_blob_bytes(header_of(e));
  return GZB_OK;
}

extern "C" int gzb_engine_export_index(gzb_engine *e, void *blob, uint64_t capacity,
                                       void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(blob, GZB_ERR_INVALID, "null blob");
  GZB_CHECK(e->have_db, GZB_ERR_INVALID, "no database chunk");
  const IndexHeader h = header_of(e);
  const uint64_t need = index_blob_bytes(h);
  GZB_CHECK(capacity >= need, GZB_ERR_INVALID, "index blob needs %llu bytes",
            (unsigned long long)need);
  cudaStream_t s = (cudaStream_t)stream;
  uint8_t *out = (uint8_t *)blob;
  memcpy(out, &h, sizeof(h));
  uint64_t at = sizeof(h), n[10];
  index_array_sizes(h, n);
  const void *src[10] = {e->X.nc_keys, e->X.nc_offsets, e->X.nc_values, e->X.rep_keys,
                         e->X.rep_offsets, e->X.rep_positions, e->X.rep_cluster_ids,
                         e->X.rep_windows, e->X.member_offsets, e->X.member_positions};
  for (int i = 0; i < 10; ++i) {
    const uint64_t bytes = n[i] * (i == 7 ? 8 : 4);
    if (bytes) GZB_CUDA(cudaMemcpyAsync(out + at, src[i], bytes, cudaMemcpyDeviceToHost, s));
    at += pad8(bytes);
  }
  GZB_CUDA(cudaStreamSynchronize(s));
  return GZB_OK;
}

extern "C" int gzb_engine_set_database_with_index(gzb_engine *e, int32_t chunk_id,
                                                  const uint8_t *codes, uint64_t length,
                                                  const uint32_t *offsets,
                                                  uint32_t number_sequences, const void *blob,
                                                  uint64_t blob_bytes, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_params, GZB_ERR_INVALID, "set_params first");
  GZB_CHECK(codes && offsets && number_sequences > 0 && length > 0 && blob, GZB_ERR_INVALID,
            "empty database or index");
  GZB_CHECK(length < (1ull << 31), GZB_ERR_OVERFLOW,
            "database chunk of %llu residues exceeds 2^31", (unsigned long long)length);
  GZB_CHECK(blob_bytes >= sizeof(IndexHeader), GZB_ERR_INVALID, "index blob too short");
  IndexHeader h;
  memcpy(&h, blob, sizeof(h));
  GZB_CHECK(h.magic == kIndexMagic, GZB_ERR_INVALID, "not an index blob of this library");
  GZB_CHECK(h.fingerprint == index_fingerprint(e), GZB_ERR_INVALID,
            "index blob was built with other index parameters");
  GZB_CHECK(h.db_len == length && h.nseq == number_sequences &&
                h.db_check == db_check(codes, length, offsets, number_sequences),
            GZB_ERR_INVALID, "index blob belongs to another chunk");
  GZB_CHECK(blob_bytes >= index_blob_bytes(h), GZB_ERR_INVALID, "index blob truncated");
  cudaStream_t s = (cudaStream_t)stream;
  e->have_db = false;
  e->x_in_arrays = false;
  e->chunk_id = chunk_id;
  e->db_len = length;
  e->nseq = number_sequences;
  e->db_check = h.db_check;
  GZB_TRY(upload_padded(e->db_buf, e->codeflag, codes, length, (uint8_t)e->params.delimiter, s));
  GZB_TRY(upload(e->db_offsets, offsets, number_sequences + 1, s));
  std::vector<DBuf> &B = e->index_bufs;
  uint64_t n[10], at = sizeof(h);
  index_array_sizes(h, n);
  void *dst[10];
  for (int i = 0; i < 10; ++i) {
    const uint64_t bytes = n[i] * (i == 7 ? 8 : 4);
    DBuf &d = B[40 + i];
    GZB_TRY(d.ensure(bytes + 16));
    GZB_CUDA(cudaMemsetAsync(d.p, 0, 16, s));
    if (bytes)
      GZB_CUDA(cudaMemcpyAsync(d.p, (const uint8_t *)blob + at, bytes, cudaMemcpyHostToDevice, s));
    dst[i] = d.p;
    at += pad8(bytes);
  }
  DevIndex &X = e->X;
  X = DevIndex();
  X.nc_keys = (uint32_t *)dst[0];
  X.nc_offsets = (uint32_t *)dst[1];
  X.nc_values = (uint32_t *)dst[2];
  X.rep_keys = (uint32_t *)dst[3];
  X.rep_offsets = (uint32_t *)dst[4];
  X.rep_positions = (uint32_t *)dst[5];
  X.rep_cluster_ids = (uint32_t *)dst[6];
  X.rep_windows = (uint64_t *)dst[7];
  X.member_offsets = (uint32_t *)dst[8];
  X.member_positions = (uint32_t *)dst[9];
  X.n_nc_keys = h.n_nc_keys;
  X.n_nc_values = h.n_nc_values;
  X.n_rep_keys = h.n_rep_keys;
  X.n_reps = h.n_reps;
  X.n_members = h.n_members;
  X.params_clustering = e->params.clustering != 0;
  GZB_CUDA(cudaStreamSynchronize(s));
  e->x_in_arrays = true;
  e->have_db = true;
  return GZB_OK;
}

namespace {

constexpr uint32_t kMaxDbSlots = 64;

// validates an index blob against the engine's parameters and a chunk
int check_index_blob(gzb_engine *e, const uint8_t *codes, uint64_t length,
                     const uint32_t *offsets, uint32_t number_sequences, const void *blob,
                     uint64_t blob_bytes, IndexHeader *out) {
  GZB_CHECK(codes && offsets && number_sequences > 0 && length > 0 && blob, GZB_ERR_INVALID,
            "empty database or index");
  GZB_CHECK(length < (1ull << 31), GZB_ERR_OVERFLOW,
            "database chunk of %llu residues exceeds 2^31", (unsigned long long)length);
  GZB_CHECK(blob_bytes >= sizeof(IndexHeader), GZB_ERR_INVALID, "index blob too short");
  IndexHeader h;
  memcpy(&h, blob, sizeof(h));
  GZB_CHECK(h.magic == kIndexMagic, GZB_ERR_INVALID, "not an index blob of this library");
  GZB_CHECK(h.fingerprint == index_fingerprint(e), GZB_ERR_INVALID,
            "index blob was built with other index parameters");
  GZB_CHECK(h.db_len == length && h.nseq == number_sequences &&
                h.db_check == db_check(codes, length, offsets, number_sequences),
            GZB_ERR_INVALID, "index blob belongs to another chunk");
  GZB_CHECK(blob_bytes >= index_blob_bytes(h), GZB_ERR_INVALID, "index blob truncated");
  *out = h;
  return GZB_OK;
}

// X over ten index arrays of a header's sizes
void point_index(DevIndex &X, void *const dst[10], const IndexHeader &h, bool clustering) {
  X = DevIndex();
  X.nc_keys = (uint32_t *)dst[0];
  X.nc_offsets = (uint32_t *)dst[1];
  X.nc_values = (uint32_t *)dst[2];
  X.rep_keys = (uint32_t *)dst[3];
  X.rep_offsets = (uint32_t *)dst[4];
  X.rep_positions = (uint32_t *)dst[5];
  X.rep_cluster_ids = (uint32_t *)dst[6];
  X.rep_windows = (uint64_t *)dst[7];
  X.member_offsets = (uint32_t *)dst[8];
  X.member_positions = (uint32_t *)dst[9];
  X.n_nc_keys = h.n_nc_keys;
  X.n_nc_values = h.n_nc_values;
  X.n_rep_keys = h.n_rep_keys;
  X.n_reps = h.n_reps;
  X.n_members = h.n_members;
  X.params_clustering = clustering;
}

// moves the resident chunk's index arrays into index_bufs[40..49] (device
// copies), so that the chunk can be stored without the build's scratch
int compact_index(gzb_engine *e, cudaStream_t s) {
  const IndexHeader h = header_of(e);
  uint64_t n[10];
  index_array_sizes(h, n);
  const void *src[10] = {e->X.nc_keys, e->X.nc_offsets, e->X.nc_values, e->X.rep_keys,
                         e->X.rep_offsets, e->X.rep_positions, e->X.rep_cluster_ids,
                         e->X.rep_windows, e->X.member_offsets, e->X.member_positions};
  void *dst[10];
  for (int i = 0; i < 10; ++i) {
    const uint64_t bytes = n[i] * (i == 7 ? 8 : 4);
    DBuf &d = e->index_bufs[40 + i];
    GZB_TRY(d.ensure(bytes + 16));
    GZB_CUDA(cudaMemsetAsync(d.p, 0, 16, s));
    if (bytes) GZB_CUDA(cudaMemcpyAsync(d.p, src[i], bytes, cudaMemcpyDeviceToDevice, s));
    dst[i] = d.p;
  }
  GZB_CUDA(cudaStreamSynchronize(s));
  point_index(e->X, dst, h, e->X.params_clustering);
  e->x_in_arrays = true;
  return GZB_OK;
}

}  // namespace

extern "C" int gzb_engine_swap_database(gzb_engine *e, uint32_t slot, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(slot < kMaxDbSlots, GZB_ERR_INVALID, "database slot %u outside 0..%u", slot,
            kMaxDbSlots - 1);
  if (slot >= e->db_slots.size()) e->db_slots.resize(slot + 1);
  gzb_engine::DbSlot &S = e->db_slots[slot];
  cudaStream_t s = (cudaStream_t)stream;
  if (S.pending) {
    // a prefetched chunk: its copies must be done and its codes valid
    GZB_CUDA(cudaEventSynchronize(S.ready));
    S.pending = false;
    unsigned int bad = 0;
    GZB_CUDA(cudaMemcpy(&bad, S.codeflag.p, 4, cudaMemcpyDeviceToHost));
    if (bad) {
      S.have = false;
      return set_error(GZB_ERR_INVALID, "prefetched chunk: residue codes must be below 32");
    }
  }
  if (e->have_db && !e->x_in_arrays) GZB_TRY(compact_index(e, s));
  // work already queued on `stream` may still read the resident chunk
  GZB_CUDA(cudaStreamSynchronize(s));
  std::swap(e->db_buf, S.db_buf);
  std::swap(e->db_offsets, S.db_offsets);
  std::swap(e->codeflag, S.codeflag);
  for (int i = 0; i < 10; ++i) std::swap(e->index_bufs[40 + i], S.arrays[i]);
  std::swap(e->chunk_id, S.chunk_id);
  std::swap(e->db_len, S.db_len);
  std::swap(e->db_check, S.db_check);
  std::swap(e->nseq, S.nseq);
  std::swap(e->X, S.X);
  const bool had = e->have_db;
  e->have_db = S.have;
  S.have = had;
  e->x_in_arrays = e->have_db;
  return GZB_OK;
}

extern "C" int gzb_engine_prefetch_database_with_index(
    gzb_engine *e, uint32_t slot, int32_t chunk_id, const uint8_t *codes, uint64_t length,
    const uint32_t *offsets, uint32_t number_sequences, const void *blob, uint64_t blob_bytes,
    void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_params, GZB_ERR_INVALID, "set_params first");
  GZB_CHECK(slot < kMaxDbSlots, GZB_ERR_INVALID, "database slot %u outside 0..%u", slot,
            kMaxDbSlots - 1);
  IndexHeader h;
  GZB_TRY(check_index_blob(e, codes, length, offsets, number_sequences, blob, blob_bytes, &h));
  if (slot >= e->db_slots.size()) e->db_slots.resize(slot + 1);
  gzb_engine::DbSlot &S = e->db_slots[slot];
  if (S.pending) GZB_CUDA(cudaEventSynchronize(S.ready));
  if (!S.ready) GZB_CUDA(cudaEventCreateWithFlags(&S.ready, cudaEventDisableTiming));
  cudaStream_t s = (cudaStream_t)stream;
  S.have = false;
  S.pending = false;
  // codes with their padding, and the range check that the swap reads
  GZB_TRY(S.db_buf.ensure(length + 2 * kPad));
  GZB_TRY(S.codeflag.ensure(4));
  const uint8_t delim = (uint8_t)e->params.delimiter;
  GZB_CUDA(cudaMemsetAsync(S.db_buf.p, delim, kPad, s));
  GZB_CUDA(cudaMemsetAsync((uint8_t *)S.db_buf.p + kPad + length, delim, kPad, s));
  GZB_CUDA(cudaMemcpyAsync((uint8_t *)S.db_buf.p + kPad, codes, length, cudaMemcpyHostToDevice,
                           s));
  GZB_CUDA(cudaMemsetAsync(S.codeflag.p, 0, 4, s));
  code_range_kernel<<<grid1(length / 16 + 1, 256), 256, 0, s>>>(
      (const uint8_t *)S.db_buf.p + kPad, length, S.codeflag.as<unsigned int>());
  GZB_CUDA(cudaGetLastError());
  GZB_TRY(upload(S.db_offsets, offsets, number_sequences + 1, s));
  uint64_t n[10], at = sizeof(h);
  index_array_sizes(h, n);
  void *dst[10];
  for (int i = 0; i < 10; ++i) {
    const uint64_t bytes = n[i] * (i == 7 ? 8 : 4);
    DBuf &d = S.arrays[i];
    GZB_TRY(d.ensure(bytes + 16));
    GZB_CUDA(cudaMemsetAsync(d.p, 0, 16, s));
    if (bytes)
      GZB_CUDA(cudaMemcpyAsync(d.p, (const uint8_t *)blob + at, bytes, cudaMemcpyHostToDevice, s));
    dst[i] = d.p;
    at += pad8(bytes);
  }
  point_index(S.X, dst, h, e->params.clustering != 0);
  S.chunk_id = chunk_id;
  S.db_len = length;
  S.nseq = number_sequences;
  S.db_check = h.db_check;
  GZB_CUDA(cudaEventRecord(S.ready, s));
  S.pending = true;
  S.have = true;
  return GZB_OK;
}

namespace {
// The device side of a new query set whose codes, offsets, lengths, cutoffs
// and triggers are on the device: nearest delimiters, the hash lists
// (SeedSearcherGpuQueryParameters::Build) and empty results.
int build_query_lists(gzb_engine *e, uint64_t length, uint32_t number_queries, cudaStream_t s) {
  GZB_TRY(e->q_prev.ensure(4 * (length + 1)));
  GZB_TRY(e->q_next.ensure(4 * (length + 1)));
  delim_dist_kernel<<<grid1((uint64_t)number_queries * 32, 256), 256, 0, s>>>(
      e->q_buf.as<uint8_t>() + kPad, e->q_offsets.as<uint32_t>(), e->q_lengths.as<uint32_t>(),
      number_queries, e->params.delimiter, e->q_prev.as<uint32_t>(), e->q_next.as<uint32_t>());
  GZB_CUDA(cudaGetLastError());
  std::vector<DBuf> &B = e->list_bufs;
  DBuf &keys = B[0], &alt = B[1];
  GZB_TRY(keys.ensure(8 * (length + 1)));
  GZB_TRY(alt.ensure(8 * (length + 1)));
  GZB_TRY(e->ctr.ensure(64));
  GZB_CUDA(cudaMemsetAsync(e->ctr.p, 0, 8, s));
  query_entries_kernel<<<grid1((uint64_t)number_queries * 32, 256), 256, 0, s>>>(
      e->dp, e->q_buf.as<uint8_t>() + kPad, e->q_offsets.as<uint32_t>(),
      e->q_lengths.as<uint32_t>(), e->q_prev.as<uint32_t>(), e->q_next.as<uint32_t>(),
      number_queries, keys.as<uint64_t>(), e->ctr.as<unsigned long long>(), length + 1);
  GZB_CUDA(cudaGetLastError());
  uint64_t n = 0;
  GZB_CUDA(cudaMemcpyAsync(&n, e->ctr.p, 8, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  uint64_t *sorted = nullptr;
  GZB_TRY(sort_keys_u64(e, keys.as<uint64_t>(), alt.as<uint64_t>(), n, 64, s, &sorted));
  DBuf &flags = B[2], &starts = B[3];
  GZB_TRY(flags.ensure(n + 1));
  GZB_TRY(starts.ensure(4 * (n + 1)));
  uint64_t nl = 0;
  if (n) {
    key_start_flags<<<grid1(n, 256), 256, 0, s>>>(sorted, n, flags.as<uint8_t>());
    GZB_CUDA(cudaGetLastError());
    GZB_TRY(select_flagged_index(e, flags.as<uint8_t>(), n, starts.as<uint32_t>(), &nl, s));
  }
  DevLists &L = e->L;
  L = DevLists();
  DBuf *bufs[] = {&B[4], &B[5], &B[6], &B[7], &B[8], &B[9], &B[10], &B[11], &B[12], &B[13]};
  GZB_TRY(B[4].ensure(4 * (nl + 1)));   // hash
  GZB_TRY(B[5].ensure(4 * (nl + 2)));   // offsets
  GZB_TRY(B[6].ensure(4 * (nl + 1)));   // nchk
  GZB_TRY(B[7].ensure(4 * (nl + 1)));   // rep_begin
  GZB_TRY(B[8].ensure(4 * (nl + 1)));   // rep_count
  GZB_TRY(B[9].ensure(4 * (nl + 1)));   // nc_begin
  GZB_TRY(B[10].ensure(4 * (nl + 1)));  // nc_count
  GZB_TRY(B[11].ensure(8 * (nl + 2)));  // unit offsets
  GZB_TRY(B[12].ensure(4 * (n + 1)));   // entry qid
  GZB_TRY(B[13].ensure(4 * (n + 1)));   // entry cpos
  (void)bufs;
  L.hash = B[4].as<uint32_t>();
  L.offsets = B[5].as<uint32_t>();
  L.nchk = B[6].as<uint32_t>();
  L.rep_begin = B[7].as<uint32_t>();
  L.rep_count = B[8].as<uint32_t>();
  L.nc_begin = B[9].as<uint32_t>();
  L.nc_count = B[10].as<uint32_t>();
  L.unit_offsets = B[11].as<uint64_t>();
  L.entry_qid = B[12].as<uint32_t>();
  L.entry_cpos = B[13].as<uint32_t>();
  L.n_lists = nl;
  L.n_entries = n;
  GZB_TRY(B[16].ensure(8 * (n + 1)));
  L.entry_window = B[16].as<uint64_t>();
  GZB_TRY(B[17].ensure(4 * (n + 1)));
  L.entry_ct = B[17].as<uint32_t>();
  if (n) {
    list_fill_kernel<<<grid1(n + nl + 1, 256), 256, 0, s>>>(
        sorted, n, starts.as<uint32_t>(), nl, e->q_offsets.as<uint32_t>(), number_queries,
        L.hash, L.offsets, L.nchk, L.entry_qid, L.entry_cpos);
    GZB_CUDA(cudaGetLastError());
    entry_window_kernel<<<grid1(n, 256), 256, 0, s>>>(
        e->dp, e->q_buf.as<uint8_t>() + kPad, L.entry_cpos, L.entry_qid,
        e->q_cut.as<int32_t>(), e->q_trig.as<int32_t>(), n, L.entry_window, L.entry_ct);
    GZB_CUDA(cudaGetLastError());
  } else {
    GZB_CUDA(cudaMemsetAsync(L.offsets, 0, 8, s));
  }
  // results of a new query set start empty
  GZB_TRY(e->results.ensure(sizeof(gzb_result) * (uint64_t)number_queries *
                            e->params.max_number_results));
  GZB_TRY(e->counts.ensure(4 * (uint64_t)number_queries));
  GZB_CUDA(cudaMemsetAsync(e->counts.p, 0, 4 * (uint64_t)number_queries, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  e->have_queries = true;
  return GZB_OK;
}
}  // namespace

extern "C" int gzb_engine_set_queries(
gzb_engine *e, const uint8_t *codes, uint64_t length,
                                      const uint32_t *offsets, const uint32_t *lengths,
                                      uint32_t number_queries, const int32_t *cutoffs,
                                      const int32_t *triggers, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_params, GZB_ERR_INVALID, "set_params first");
  GZB_CHECK(codes && offsets && lengths && cutoffs && triggers && number_queries > 0,
            GZB_ERR_INVALID, "empty query set");
  GZB_CHECK(length < (1ull << 31), GZB_ERR_OVERFLOW, "query buffer exceeds 2^31 residues");
  cudaStream_t s = (cudaStream_t)stream;
  e->have_queries = false;
  uint32_t maxl = 0;
  for (uint32_t i = 0; i < number_queries; ++i) {
    GZB_CHECK(lengths[i] >= 2 && (uint64_t)offsets[i] + lengths[i] <= length, GZB_ERR_INVALID,
              "query %u outside the buffer", i);
    GZB_CHECK(i == 0 || offsets[i] + 1 >= offsets[i - 1] + lengths[i - 1], GZB_ERR_INVALID,
              "query %u overlaps the previous one beyond their shared delimiter", i);
    GZB_CHECK(codes[offsets[i]] == e->params.delimiter &&
                  codes[offsets[i] + lengths[i] - 1] == e->params.delimiter,
              GZB_ERR_INVALID, "query %u does not start and end with the delimiter", i);
    GZB_CHECK(cutoffs[i] >= 1 && cutoffs[i] <= 32767, GZB_ERR_INVALID,
              "ungapped cutoff of query %u outside 1..32767", i);
    GZB_CHECK(triggers[i] >= -32768 && triggers[i] <= 32767, GZB_ERR_INVALID,
              "gapped trigger of query %u outside int16", i);
    maxl = std::max(maxl, lengths[i]);
  }
  e->nq = number_queries;
  e->q_len = length;
  e->max_qlen = maxl;
  GZB_TRY(upload_padded(e->q_buf, e->codeflag, codes, length, (uint8_t)e->params.delimiter, s));
  GZB_TRY(upload(e->q_offsets, offsets, number_queries, s));
  GZB_TRY(upload(e->q_lengths, lengths, number_queries, s));
  GZB_TRY(upload(e->q_cut, cutoffs, number_queries, s));
  GZB_TRY(upload(e->q_trig, triggers, number_queries, s));
  return build_query_lists(e, length, number_queries, s);
}

extern "C" int gzb_engine_set_protein_queries(gzb_engine *e, const uint8_t *codes,
                                              uint64_t length, const uint32_t *offsets,
                                              const uint32_t *lengths, uint32_t number_queries,
                                              int filter, float ungapped_bits,
                                              float trigger_bits, int32_t *cutoffs,
                                              int32_t *triggers, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_params, GZB_ERR_INVALID, "set_params first");
  GZB_CHECK(codes && offsets && lengths && number_queries > 0, GZB_ERR_INVALID,
            "empty query set");
  GZB_CHECK(length < (1ull << 31), GZB_ERR_OVERFLOW, "query buffer exceeds 2^31 residues");
  cudaStream_t s = (cudaStream_t)stream;
  e->have_queries = false;
  uint32_t maxl = 0;
  std::vector<uint64_t> off64(number_queries);
  std::vector<uint32_t> short_ids;
  for (uint32_t i = 0; i < number_queries; ++i) {
    GZB_CHECK(lengths[i] >= 2 && (uint64_t)offsets[i] + lengths[i] <= length, GZB_ERR_INVALID,
              "query %u outside the buffer", i);
    GZB_CHECK(i == 0 || offsets[i] + 1 >= offsets[i - 1] + lengths[i - 1], GZB_ERR_INVALID,
              "query %u overlaps the previous one beyond their shared delimiter", i);
    GZB_CHECK(codes[offsets[i]] == e->params.delimiter &&
                  codes[offsets[i] + lengths[i] - 1] == e->params.delimiter,
              GZB_ERR_INVALID, "query %u does not start and end with the delimiter", i);
    maxl = std::max(maxl, lengths[i]);
    off64[i] = offsets[i];
    // a protein the filter refuses (fewer residues than SEG's 12-letter
    // window) is held as its leading delimiter and a zero-filled body, its
    // last code 0 rather than a delimiter (ProteinQuery,
    // src/protein_query.cpp:39-49), and its statistics are those of that
    // buffer
    if (filter && lengths[i] - 2 < 12) short_ids.push_back(i);
  }
  e->nq = number_queries;
  e->q_len = length;
  e->max_qlen = maxl;
  const uint8_t delim = (uint8_t)e->params.delimiter;
  GZB_TRY(e->q_buf.ensure(length + 2 * kPad));
  GZB_TRY(e->codeflag.ensure(16));
  GZB_CUDA(cudaMemsetAsync(e->q_buf.p, delim, length + 2 * kPad, s));
  GZB_CUDA(cudaMemcpyAsync(e->q_buf.as<uint8_t>() + kPad, codes, length, cudaMemcpyHostToDevice,
                           s));
  GZB_CUDA(cudaMemsetAsync(e->codeflag.p, 0, 16, s));
  GZB_TRY(upload(e->q_offsets, offsets, number_queries, s));
  GZB_TRY(upload(e->q_lengths, lengths, number_queries, s));
  GZB_TRY(upload(e->q_off64, off64.data(), number_queries, s));
  GZB_TRY(e->q_cut.ensure(4 * (uint64_t)number_queries));
  GZB_TRY(e->q_trig.ensure(4 * (uint64_t)number_queries));
  uint8_t *q = e->q_buf.as<uint8_t>() + kPad;
  unsigned int *flags = e->codeflag.as<unsigned int>();  // codes, SEG status, cutoffs
  if (filter)
    GZB_TRY(gzb_seg_protein_queries(q, e->q_off64.as<uint64_t>(), e->q_lengths.as<uint32_t>(),
                                    number_queries, flags + 1, s));
  code_range_kernel<<<grid1(length / 16 + 1, 256), 256, 0, s>>>(q, length, flags);
  GZB_CUDA(cudaGetLastError());
  GZB_TRY(gzb_query_karlin_cutoffs(q, e->q_off64.as<uint64_t>(), e->q_lengths.as<uint32_t>(),
                                   number_queries, e->params.score_matrix,
                                   (uint32_t)e->params.number_letters, ungapped_bits,
                                   trigger_bits, e->q_cut.as<int32_t>(),
                                   e->q_trig.as<int32_t>(), nullptr, s));
  const uint32_t ns = (uint32_t)short_ids.size();
  if (ns) {
    // the short proteins' buffers, back to back, then their cutoffs
    std::vector<uint64_t> so(ns);
    std::vector<uint32_t> sl(ns);
    uint64_t total = 0;
    for (uint32_t j = 0; j < ns; ++j) {
      so[j] = total;
      sl[j] = lengths[short_ids[j]];
      total += sl[j];
    }
    std::vector<uint8_t> buf(total, 0);
    for (uint32_t j = 0; j < ns; ++j) buf[so[j]] = delim;
    const uint64_t at_idx = 0, at_off = 4 * (ns + 1) / 8 * 8 + 8, at_len = at_off + 8 * ns,
                   at_c = at_len + 4 * ns, at_t = at_c + 4 * ns, at_buf = at_t + 4 * ns;
    GZB_TRY(e->q_prep.ensure(at_buf + total + 2 * kPad));
    uint8_t *base = e->q_prep.as<uint8_t>();
    GZB_CUDA(cudaMemcpyAsync(base + at_idx, short_ids.data(), 4 * ns, cudaMemcpyHostToDevice, s));
    GZB_CUDA(cudaMemcpyAsync(base + at_off, so.data(), 8 * ns, cudaMemcpyHostToDevice, s));
    GZB_CUDA(cudaMemcpyAsync(base + at_len, sl.data(), 4 * ns, cudaMemcpyHostToDevice, s));
    GZB_CUDA(cudaMemsetAsync(base + at_buf, delim, total + 2 * kPad, s));
    GZB_CUDA(cudaMemcpyAsync(base + at_buf + kPad, buf.data(), total, cudaMemcpyHostToDevice, s));
    GZB_TRY(gzb_query_karlin_cutoffs(
        base + at_buf + kPad, reinterpret_cast<const uint64_t *>(base + at_off),
        reinterpret_cast<const uint32_t *>(base + at_len), ns, e->params.score_matrix,
        (uint32_t)e->params.number_letters, ungapped_bits, trigger_bits,
        reinterpret_cast<int32_t *>(base + at_c), reinterpret_cast<int32_t *>(base + at_t),
        nullptr, s));
    scatter_cutoffs_kernel<<<grid1(ns, 128), 128, 0, s>>>(
        reinterpret_cast<const uint32_t *>(base + at_idx),
        reinterpret_cast<const int32_t *>(base + at_c),
        reinterpret_cast<const int32_t *>(base + at_t), ns, e->q_cut.as<int32_t>(),
        e->q_trig.as<int32_t>());
    GZB_CUDA(cudaGetLastError());
  }
  cutoff_range_kernel<<<grid1(number_queries, 256), 256, 0, s>>>(
      e->q_cut.as<int32_t>(), e->q_trig.as<int32_t>(), number_queries, flags + 2);
  GZB_CUDA(cudaGetLastError());
  if (cutoffs)
    GZB_CUDA(cudaMemcpyAsync(cutoffs, e->q_cut.p, 4 * (uint64_t)number_queries,
                             cudaMemcpyDeviceToHost, s));
  if (triggers)
    GZB_CUDA(cudaMemcpyAsync(triggers, e->q_trig.p, 4 * (uint64_t)number_queries,
                             cudaMemcpyDeviceToHost, s));
  unsigned int bad[3] = {0, 0, 0};
  GZB_CUDA(cudaMemcpyAsync(bad, flags, 12, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  GZB_CHECK(bad[0] == 0, GZB_ERR_INVALID, "residue codes must be below 32 (after SEG)");
  GZB_CHECK(bad[1] == 0, GZB_ERR_INVALID, "SEG left %u queries unmasked", bad[1]);
  GZB_CHECK(bad[2] == 0, GZB_ERR_INVALID,
            "a query's cutoff is outside 1..32767 or its trigger outside int16");
  return build_query_lists(e, length, number_queries, s);
}

extern "C" int gzb_engine_set_translated_queries(gzb_engine *e, const uint8_t *dna,
                                                 const uint64_t *read_offsets,
                                                 uint32_t number_reads, int filter,
                                                 float ungapped_bits, float trigger_bits,
                                                 int32_t *cutoffs, int32_t *triggers,
                                                 void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_params, GZB_ERR_INVALID, "set_params first");
  GZB_CHECK(dna && read_offsets && number_reads > 0, GZB_ERR_INVALID, "empty read set");
  cudaStream_t s = (cudaStream_t)stream;
  e->have_queries = false;
  // the shared-delimiter layout of the six-frame queries
  const uint32_t n = number_reads;
  std::vector<uint32_t> read_len(n), qoff(n), qlen(n);
  std::vector<uint64_t> qoff64(n);
  uint64_t total = 1, maxl = 0;
  for (uint32_t r = 0; r < n; ++r) {
    GZB_CHECK(read_offsets[r + 1] >= read_offsets[r] &&
                  read_offsets[r + 1] - read_offsets[r] <= 0xFFFFFFFFull,
              GZB_ERR_INVALID, "read %u: offsets must be non-decreasing", r);
    read_len[r] = (uint32_t)(read_offsets[r + 1] - read_offsets[r]);
    const uint64_t ql = gzb_translated_query_length(read_len[r]);
    qoff64[r] = total - 1;
    total += ql - 1;
    GZB_CHECK(total < (1ull << 31), GZB_ERR_OVERFLOW,
              "translated queries exceed 2^31 codes");
    qoff[r] = (uint32_t)qoff64[r];
    qlen[r] = (uint32_t)ql;
    maxl = std::max<uint64_t>(maxl, ql);
  }
  const uint64_t bases = read_offsets[n] - read_offsets[0];
  e->nq = n;
  e->q_len = total;
  e->max_qlen = (uint32_t)maxl;
  const uint8_t delim = (uint8_t)e->params.delimiter;
  GZB_TRY(e->q_buf.ensure(total + 2 * kPad));
  GZB_TRY(e->codeflag.ensure(16));
  GZB_CUDA(cudaMemsetAsync(e->q_buf.p, delim, total + 2 * kPad, s));
  GZB_CUDA(cudaMemsetAsync(e->codeflag.p, 0, 16, s));
  // reads and their offsets (relative to the first read) after the layout
  const uint64_t at_len = ((bases + 15) / 16) * 16, at_off = at_len + ((4ull * n + 15) / 16) * 16;
  GZB_TRY(e->q_prep.ensure(at_off + 8ull * n + 16));
  uint8_t *base = e->q_prep.as<uint8_t>();
  std::vector<uint64_t> roff(n);
  for (uint32_t r = 0; r < n; ++r) roff[r] = read_offsets[r] - read_offsets[0];
  if (bases)
    GZB_CUDA(cudaMemcpyAsync(base, dna + read_offsets[0], bases, cudaMemcpyHostToDevice, s));
  GZB_CUDA(cudaMemcpyAsync(base + at_len, read_len.data(), 4ull * n, cudaMemcpyHostToDevice, s));
  GZB_CUDA(cudaMemcpyAsync(base + at_off, roff.data(), 8ull * n, cudaMemcpyHostToDevice, s));
  GZB_TRY(upload(e->q_offsets, qoff.data(), n, s));
  GZB_TRY(upload(e->q_lengths, qlen.data(), n, s));
  GZB_TRY(upload(e->q_off64, qoff64.data(), n, s));
  GZB_TRY(e->q_cut.ensure(4 * (uint64_t)n));
  GZB_TRY(e->q_trig.ensure(4 * (uint64_t)n));
  uint8_t *q = e->q_buf.as<uint8_t>() + kPad;
  const uint32_t *d_read_len = reinterpret_cast<const uint32_t *>(base + at_len);
  unsigned int *flags = e->codeflag.as<unsigned int>();  // codes, SEG status, cutoffs
  GZB_TRY(gzb_translate_dna_queries(base, reinterpret_cast<const uint64_t *>(base + at_off),
                                    d_read_len, n, e->q_off64.as<uint64_t>(), delim, q, s));
  if (filter)
    GZB_TRY(gzb_seg_translated_queries(q, e->q_off64.as<uint64_t>(), d_read_len, n, flags + 1,
                                       s));
  code_range_kernel<<<grid1(total / 16 + 1, 256), 256, 0, s>>>(q, total, flags);
  GZB_CUDA(cudaGetLastError());
  GZB_TRY(gzb_query_karlin_cutoffs(q, e->q_off64.as<uint64_t>(), e->q_lengths.as<uint32_t>(), n,
                                   e->params.score_matrix, (uint32_t)e->params.number_letters,
                                   ungapped_bits, trigger_bits, e->q_cut.as<int32_t>(),
                                   e->q_trig.as<int32_t>(), nullptr, s));
  cutoff_range_kernel<<<grid1(n, 256), 256, 0, s>>>(e->q_cut.as<int32_t>(),
                                                      e->q_trig.as<int32_t>(), n, flags + 2);
  GZB_CUDA(cudaGetLastError());
  if (cutoffs)
    GZB_CUDA(cudaMemcpyAsync(cutoffs, e->q_cut.p, 4ull * n, cudaMemcpyDeviceToHost, s));
  if (triggers)
    GZB_CUDA(cudaMemcpyAsync(triggers, e->q_trig.p, 4ull * n, cudaMemcpyDeviceToHost, s));
  unsigned int bad[3] = {0, 0, 0};
  GZB_CUDA(cudaMemcpyAsync(bad, flags, 12, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  GZB_CHECK(bad[0] == 0, GZB_ERR_INVALID, "residue codes must be below 32");
  GZB_CHECK(bad[1] == 0, GZB_ERR_INVALID, "SEG left %u frames unmasked", bad[1]);
  GZB_CHECK(bad[2] == 0, GZB_ERR_INVALID,
            "a query's cutoff is outside 1..32767 or its trigger outside int16");
  return build_query_lists(e, total, n, s);
}

extern "C" int gzb_engine_reset_results(gzb_engine *e, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_queries, GZB_ERR_INVALID, "no queries");
  GZB_CUDA(cudaMemsetAsync(e->counts.p, 0, 4 * (uint64_t)e->nq, (cudaStream_t)stream));
  return GZB_OK;
}

namespace {

// chain_kernel over the queries, one warp per block, the diagonal slots in
// shared memory for queries up to kChainSmemSlots long
int launch_chain(gzb_engine *e, uint32_t nq, uint64_t *hits, const uint64_t *begin, int qbits,
                 int dbits, uint32_t *kept, cudaStream_t s) {
  const uint32_t smem_slots = std::min<uint32_t>(e->max_qlen, kChainSmemSlots);
  const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>(nq, 148u * 64u));
  chain_kernel<<<blocks, 32, sizeof(uint2) * smem_slots, s>>>(
      e->dp, e->q_buf.as<uint8_t>() + kPad, e->db_buf.as<uint8_t>() + kPad,
      e->q_offsets.as<uint32_t>(), e->q_lengths.as<uint32_t>(), e->q_cut.as<int32_t>(),
      e->matrix32.as<int32_t>(), nq, hits, begin, qbits, dbits, e->slots.as<uint2>(), kept,
      smem_slots);
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}

int presearch_impl(gzb_engine *e, int schedule, cudaStream_t s) {
  uint64_t launches = 0;
  GappedTile stile = g_tile;
  for (int w = 0; w < kTileParameters; ++w)
    if (e->tile[schedule][w] >= 0) *tile_field(stile, w) = e->tile[schedule][w];
  DevLists &L = e->L;
  const DevIndex &X = e->X;
  const uint32_t nq = e->nq;
  GZB_CUDA(cudaEventRecord(e->ev[0], s));
  // ---- list lookup against this chunk's index
  if (L.n_lists) {
    GZB_TRY(e->list_bufs[14].ensure(8 * (L.n_lists + 1)));
    uint64_t *unit_counts = e->list_bufs[14].as<uint64_t>();
    list_lookup_kernel<<<grid1(L.n_lists, 256), 256, 0, s>>>(L, X, e->params.clustering,
                                                              unit_counts);
    GZB_CUDA(cudaGetLastError());
    ++launches;
    GZB_CUDA(cudaMemsetAsync(unit_counts + L.n_lists, 0, 8, s));
    GZB_TRY(exclusive_sum(e, unit_counts, L.unit_offsets, L.n_lists + 1, s));
    GZB_CUDA(cudaMemcpyAsync(&L.n_units, L.unit_offsets + L.n_lists, 8, cudaMemcpyDeviceToHost, s));
    GZB_CUDA(cudaStreamSynchronize(s));
  } else {
    L.n_units = 0;
  }
  GZB_CUDA(cudaEventRecord(e->ev[1], s));
  // ---- seed search + distance + ungapped with trigger
  const int qbits = bits_for(e->max_qlen);
  const int dbits = bits_for(e->db_len + 1);
  const int nqbits = bits_for(nq);
  GZB_CHECK(qbits + dbits + nqbits <= 64, GZB_ERR_OVERFLOW,
            "hit key needs %d bits (queries %u, chunk %llu, longest query %u)",
            qbits + dbits + nqbits, nq, (unsigned long long)e->db_len, e->max_qlen);
  GZB_TRY(e->ctr.ensure(64));
  uint64_t n_hits = 0, n_mwork = 0;
  unsigned long long hctr[8];
  for (int attempt = 0; attempt < 4; ++attempt) {
    GZB_TRY(e->hits.ensure(8 * e->hit_cap));
    GZB_TRY(e->mwork.ensure(8 * e->mwork_cap));
    GZB_CUDA(cudaMemsetAsync(e->ctr.p, 0, 64, s));
    SeedArgs a;
    a.p = e->dp;
    a.L = L;
    a.X = X;
    a.q = e->q_buf.as<uint8_t>() + kPad;
    a.db = e->db_buf.as<uint8_t>() + kPad;
    a.q_offsets = e->q_offsets.as<uint32_t>();
    a.cutoffs = e->q_cut.as<int32_t>();
    a.triggers = e->q_trig.as<int32_t>();
    a.matrix32 = e->matrix32.as<int32_t>();
    a.clustering = e->params.clustering;
    a.dbits = dbits;
    a.qbits = qbits;
    a.hits = e->hits.as<uint64_t>();
    unsigned long long *c = e->ctr.as<unsigned long long>();
    a.hit_count = c + 4;
    a.hit_cap = e->hit_cap;
    a.mwork = e->mwork.as<uint2>();
    a.mwork_count = c + 5;
    a.mwork_cap = e->mwork_cap;
    a.ctr = c;
    if (L.n_units) {
      const uint64_t warps = (L.n_units + kUnitsPerWarp - 1) / kUnitsPerWarp;
      if (stile.seed_walker == GZB_SEED_WALKER_DEALT)
        seed_dealt_kernel<<<grid1(warps * 32, kSeedBlock, 148 * 16), kSeedBlock, 0, s>>>(a);
      else
        seed_kernel<<<grid1(warps * 32, kSeedBlock, 148 * 16), kSeedBlock, 0, s>>>(a);
      GZB_CUDA(cudaGetLastError());
      ++launches;
    }
    GZB_CUDA(cudaMemcpyAsync(hctr, c, 64, cudaMemcpyDeviceToHost, s));
    GZB_CUDA(cudaStreamSynchronize(s));
    n_mwork = hctr[5];
    if (n_mwork > e->mwork_cap) {
      e->mwork_cap = n_mwork + n_mwork / 8 + 1024;
      continue;
    }
    if (n_mwork) {
      // cluster-major order (stable, so entries keep their order within a
      // cluster): the items a warp takes then share their members, whose
      // database words stay in cache between query positions
      GZB_TRY(e->mwork_alt.ensure(8 * (n_mwork + 1)));
      uint64_t *sorted_mw = nullptr;
      GZB_TRY(sort_keys_u64(e, reinterpret_cast<uint64_t *>(a.mwork),
                            e->mwork_alt.as<uint64_t>(), n_mwork, bits_for(X.n_reps + 1), s,
                            &sorted_mw));
      launches += 1;
      member_kernel<<<grid1((n_mwork + 31) / 32 * 32, kSeedBlock, 148 * 16), kSeedBlock, 0, s>>>(
          a, reinterpret_cast<const uint2 *>(sorted_mw), n_mwork, nullptr);
      GZB_CUDA(cudaGetLastError());
      ++launches;
      GZB_CUDA(cudaMemcpyAsync(hctr, c, 64, cudaMemcpyDeviceToHost, s));
      GZB_CUDA(cudaStreamSynchronize(s));
    }
    n_hits = hctr[4];
    if (n_hits > e->hit_cap) {
      e->hit_cap = n_hits + n_hits / 8 + 1024;
      continue;
    }
    break;
  }
  GZB_CHECK(n_hits <= e->hit_cap && n_mwork <= e->mwork_cap, GZB_ERR_OVERFLOW,
            "seed buffers did not converge");
  e->counters.distance_seeds = hctr[0];
  e->counters.ungapped_steps = hctr[2];
  e->counters.ungapped_seeds = hctr[1];
  e->counters.ungapped_hits = n_hits;
  GZB_CUDA(cudaEventRecord(e->ev[6], s));
  // ---- sort hits by (query, database position, query position)
  GZB_TRY(e->hits_alt.ensure(8 * (n_hits + 1)));
  uint64_t *hits = e->hits.as<uint64_t>();
  if (n_hits) {
    uint64_t *sorted = nullptr;
    GZB_TRY(sort_keys_u64(e, hits, e->hits_alt.as<uint64_t>(), n_hits,
                          qbits + dbits + nqbits, s, &sorted));
    hits = sorted;
  }
  GZB_TRY(e->hits_copy.ensure(8 * (n_hits + 1)));
  if (n_hits)
    GZB_CUDA(cudaMemcpyAsync(e->hits_copy.p, hits, 8 * n_hits, cudaMemcpyDeviceToDevice, s));
  e->qbits = qbits;
  e->dbits = dbits;
  GZB_CUDA(cudaEventRecord(e->ev[2], s));
  // ---- chain filter
  GZB_TRY(e->begin.ensure(8 * (nq + 1)));
  GZB_TRY(e->kept.ensure(4 * (nq + 1)));
  GZB_TRY(e->surv_off.ensure(8 * (nq + 1)));
  GZB_TRY(e->slots.ensure(8 * (e->q_len + nq + 1)));
  uint64_t *begin = e->begin.as<uint64_t>();
  uint32_t *kept = e->kept.as<uint32_t>();
  uint64_t *surv_off = e->surv_off.as<uint64_t>();
  hit_segments_kernel<<<grid1(nq + 1, 256), 256, 0, s>>>(hits, n_hits, nq, qbits + dbits, begin,
                                                          nullptr);
  GZB_CUDA(cudaGetLastError());
    ++launches;
  GZB_TRY(launch_chain(e, nq, hits, begin, qbits, dbits, kept, s));
  GZB_CUDA(cudaGetLastError());
    ++launches;
  GZB_CUDA(cudaMemsetAsync(kept + nq, 0, 4, s));
  GZB_TRY(exclusive_sum(e, kept, surv_off, nq + 1, s));
  uint64_t n_surv = 0;
  GZB_CUDA(cudaMemcpyAsync(&n_surv, surv_off + nq, 8, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  e->counters.chained_hits = n_surv;
  GZB_CUDA(cudaEventRecord(e->ev[3], s));
  // ---- gapped extension, both sides
  const uint64_t next = 2 * n_surv;
  GZB_TRY(e->eq.ensure(4 * (next + 1)));
  GZB_TRY(e->ed.ensure(4 * (next + 1)));
  GZB_TRY(e->edir.ensure(next + 1));
  GZB_TRY(e->escore.ensure(4 * (next + 1)));
  GZB_TRY(e->elen0.ensure(4 * (next + 1)));
  GZB_TRY(e->elen1.ensure(4 * (next + 1)));
  GZB_TRY(e->eqid.ensure(4 * (next + 1)));
  GZB_TRY(e->enb.ensure(4 * (n_surv + 1)));
  e->last_mae = -1.0f;
  e->last_mae_n = 0;
  e->pred_n = 0;
  if (n_surv) {
    GappedTile tile = g_tile;
    for (int w = 0; w < kTileParameters; ++w)
      if (e->tile[schedule][w] >= 0) *tile_field(tile, w) = e->tile[schedule][w];
    if (schedule == GZB_SCHEDULE_PLAIN) tile.kernel = GZB_GAPPED_KERNEL_STATIC;
    const bool learned =
        schedule == GZB_SCHEDULE_BATCHED && e->have_model && tile.order == GZB_ORDER_MODEL;
    const bool oracle_order = schedule == GZB_SCHEDULE_ORACLE && e->prev_cells_n == next;
    const bool scheduled = schedule != GZB_SCHEDULE_PLAIN || e->logging;
    const bool want_feat = learned || e->logging;
    build_ext_kernel<<<grid1((uint64_t)nq * 32, 256), 256, 0, s>>>(
        hits, begin, kept, surv_off, nq, e->q_offsets.as<uint32_t>(),
        e->q_lengths.as<uint32_t>(), e->db_offsets.as<uint32_t>(), e->nseq, (uint32_t)e->db_len,
        qbits, dbits, n_surv, e->eq.as<uint32_t>(), e->ed.as<uint32_t>(), e->edir.as<uint8_t>(),
        e->elen0.as<uint32_t>(), e->elen1.as<uint32_t>(), e->eqid.as<uint32_t>(),
        e->enb.as<uint32_t>(), nullptr, e->q_prev.as<uint32_t>(), e->q_next.as<uint32_t>(),
        want_feat ? 1 : 0);
    GZB_CUDA(cudaGetLastError());
    ++launches;
    GZB_CUDA(cudaMemsetAsync(e->gcells, 0, 8, s));
    GappedJob job;
    job.query = e->q_buf.as<uint8_t>() + kPad;
    job.db = e->db_buf.as<uint8_t>() + kPad;
    job.delim = e->params.delimiter;
    job.gap_open = e->params.gap_open;
    job.gap_ext = e->params.gap_extension;
    job.cutoff = e->params.gapped_cutoff;
    if (want_feat) {
      GZB_TRY(e->efeat.ensure(4 * kFeat * (next + 1)));
      ext_features_kernel<<<grid1(n_surv, 256), 256, 0, s>>>(
          job.query, job.db, job.delim, e->matrix32.as<int32_t>(), e->q_cut.as<int32_t>(),
          n_surv, e->eq.as<uint32_t>(), e->ed.as<uint32_t>(), e->elen0.as<uint32_t>(),
          e->elen1.as<uint32_t>(), e->eqid.as<uint32_t>(), e->enb.as<uint32_t>(),
          e->efeat.as<float>(), nullptr);
      GZB_CUDA(cudaGetLastError());
      ++launches;
    }
    const uint32_t *order = nullptr;
    if (learned || oracle_order) {
      GZB_TRY(e->okeys.ensure(4 * (next + 1)));
      GZB_TRY(e->okeys2.ensure(4 * (next + 1)));
      GZB_TRY(e->oidx.ensure(4 * (next + 1)));
      GZB_TRY(e->oidx2.ensure(4 * (next + 1)));
      if (learned) {
        GZB_TRY(e->epred.ensure(4 * (next + 1)));
        GZB_TRY(cost_predict(e->model_d.as<float>(), e->efeat.as<float>(), (uint32_t)next,
                             e->epred.as<float>(), s, nullptr));
        e->pred_n = next;
        ++launches;
      }
      cost_keys_kernel<<<grid1(next, 256), 256, 0, s>>>(
          learned ? e->epred.as<float>() : nullptr, e->prev_cells.as<uint32_t>(), next,
          e->okeys.as<uint32_t>(), e->oidx.as<uint32_t>(), nullptr, 0);
      GZB_CUDA(cudaGetLastError());
      ++launches;
      cub::DoubleBuffer<uint32_t> kb(e->okeys.as<uint32_t>(), e->okeys2.as<uint32_t>());
      cub::DoubleBuffer<uint32_t> vb(e->oidx.as<uint32_t>(), e->oidx2.as<uint32_t>());
      size_t tb = 0;
      GZB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb, (int64_t)next, 0, 16, s));
      GZB_TRY(e->tmp.ensure(tb));
      GZB_CUDA(cub::DeviceRadixSort::SortPairs(e->tmp.p, tb, kb, vb, (int64_t)next, 0, 16, s));
      order = vb.Current();
    }
    uint32_t fb = 0;
    if (scheduled) GZB_TRY(e->ecells.ensure(4 * (next + 1)));
    GZB_TRY(run_gapped(tile, job, e->matrix32.as<int32_t>(), 32, 32, next, order, 0,
                       e->edir.as<uint8_t>(), e->eq.as<uint32_t>(), e->ed.as<uint32_t>(),
                       e->escore.as<int32_t>(), &e->spill, &e->spill_cap, e->gcounters,
                       e->gcells, scheduled ? e->ecells.as<uint32_t>() : nullptr,
                       &e->band_pool, &e->band_wmask, s, &fb, nullptr));
    launches += 3;
    if (scheduled) {
      if (e->logging) {
        log_pairs_kernel<<<grid1(next, 256), 256, 0, s>>>(
            e->efeat.as<float>(), e->ecells.as<uint32_t>(), next, e->log_x.as<float>(),
            e->log_y.as<float>(), e->log_ctr.as<unsigned long long>(), e->log_cap);
        GZB_CUDA(cudaGetLastError());
        ++launches;
      }
      if (learned) {
        GZB_TRY(e->mae_acc.ensure(16));
        GZB_CUDA(cudaMemsetAsync(e->mae_acc.p, 0, 16, s));
        abs_error_kernel<<<grid1(next, 256), 256, 0, s>>>(e->epred.as<float>(),
                                                          e->ecells.as<uint32_t>(), next,
                                                          e->mae_acc.as<double>());
        GZB_CUDA(cudaGetLastError());
        ++launches;
        double acc[2] = {0, 0};
        GZB_CUDA(cudaMemcpyAsync(acc, e->mae_acc.p, 16, cudaMemcpyDeviceToHost, s));
        GZB_CUDA(cudaStreamSynchronize(s));
        e->last_mae = acc[1] > 0 ? (float)(acc[0] / acc[1]) : -1.0f;
        e->last_mae_n = (uint64_t)acc[1];
      }
      // true costs of this extension list, for a later oracle-ordered run
      GZB_TRY(e->prev_cells.ensure(4 * (next + 1)));
      GZB_CUDA(cudaMemcpyAsync(e->prev_cells.p, e->ecells.p, 4 * next, cudaMemcpyDeviceToDevice,
                               s));
      e->prev_cells_n = next;
    }
    unsigned long long cells = 0;
    GZB_CUDA(cudaMemcpyAsync(&cells, e->gcells, 8, cudaMemcpyDeviceToHost, s));
    GZB_CUDA(cudaStreamSynchronize(s));
    e->counters.gapped_cells = cells;
    e->counters.gapped_fallbacks = fb;
  } else {
    e->counters.gapped_cells = 0;
    e->counters.gapped_fallbacks = 0;
  }
  e->counters.gapped_extensions = next;
  GZB_CUDA(cudaEventRecord(e->ev[4], s));
  // ---- top-b merge
  if (n_surv) {
    // per candidate: its sort key (16 B), then its heap slot (4 B)
    GZB_TRY(e->heap.ensure(20 * (n_surv + 1)));
    merge_kernel<<<grid1((uint64_t)nq * 32, 128), 128, 0, s>>>(
        nq, hits, begin, kept, surv_off, n_surv, e->eq.as<uint32_t>(), e->ed.as<uint32_t>(),
        e->escore.as<int32_t>(), e->q_offsets.as<uint32_t>(), qbits, dbits,
        e->db_offsets.as<uint32_t>(), e->nseq, (uint32_t)e->db_len, e->chunk_id,
        e->params.max_number_results, e->params.max_number_one_subject_results,
        e->heap.as<ulonglong2>(),
        reinterpret_cast<uint32_t *>(e->heap.as<ulonglong2>() + n_surv + 1),
        e->results.as<gzb_result>(), e->counts.as<uint32_t>(), nullptr, nullptr);
    GZB_CUDA(cudaGetLastError());
    ++launches;
  }
  GZB_CUDA(cudaEventRecord(e->ev[5], s));
  GZB_CUDA(cudaEventSynchronize(e->ev[5]));
  float t[6];
  for (int i = 0; i < 5; ++i) GZB_CUDA(cudaEventElapsedTime(&t[i], e->ev[i], e->ev[i + 1]));
  GZB_CUDA(cudaEventElapsedTime(&t[5], e->ev[0], e->ev[5]));
  for (int i = 0; i < 6; ++i) e->stage_ms[i] = t[i];
  GZB_CUDA(cudaEventElapsedTime(&e->stage_ms[6], e->ev[1], e->ev[6]));
  e->counters.kernel_launches = launches;
  return GZB_OK;
}

// ---- graph mode: the whole presearch of the resident chunk as one CUDA
// graph.  Every count comes from device memory and every buffer is sized
// to a capacity chosen beforehand (hits, member work and the extensions
// they imply), so nothing reads back between stages; sorts run over the
// whole capacity with keys past the count set to all ones (they sort last,
// and the sorts are stable, so the first `count` keys come out as the
// eager path's).  A count above its capacity sets an overflow bit: the
// merge then does nothing, and the host redoes the call eagerly with
// larger capacities.

// count clamped to a capacity; an excess sets `bit` in *overflow
__global__ void clamp_count_kernel(const unsigned long long *count, uint64_t cap, uint64_t *out,
                                   uint32_t *overflow, uint32_t bit) {
  const unsigned long long c = *count;
  *out = c < cap ? c : cap;
  if (c > cap) atomicOr(overflow, bit);
}

// keys[n .. cap) = all ones (n read on the device)
__global__ void pad_keys_kernel(uint64_t *keys, const uint64_t *n_dev, uint64_t cap) {
  for (uint64_t i = *n_dev + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap;
       i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = ~0ull;
}

// surviving hits and the extensions they make
__global__ void ext_count_kernel(const uint64_t *surv_off, uint32_t nq, uint64_t *plan) {
  plan[2] = surv_off[nq];
  plan[3] = 2 * surv_off[nq];
}

// the device clock (ns) when the stream reaches this point: stage times of
// a graph run (events recorded inside a graph cannot be timed)
__global__ void stamp_kernel(uint64_t *t) {
  uint64_t v;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
  *t = v;
}

// everything the host reads after a graph run, in one place
__global__ void report_kernel(const unsigned long long *ctr, const uint64_t *plan,
                              const unsigned long long *gcells, const uint32_t *gcounters,
                              uint64_t *report) {
  for (int i = 0; i < 6; ++i) report[i] = ctr[i];
  report[6] = plan[2];
  report[7] = *gcells;
  report[8] = gcounters[0];
  report[9] = gcounters[1];
  report[10] = gcounters[2];
  report[11] = reinterpret_cast<const uint32_t *>(plan + 6)[0];
  report[12] = plan[1];
}

constexpr int kGraphCache = 16;        // graphs kept per engine
constexpr int kReportWords = 24;   // plan[8..31]: report, then the stage stamps

struct GraphCaps {
  uint64_t hits, mwork, ext;           // ext = 2 * hits (every hit may survive)
};

GraphCaps graph_caps(const gzb_engine *e) {
  GraphCaps c;
  c.hits = e->hit_cap;
  c.mwork = e->mwork_cap;
  c.ext = 2 * c.hits;
  return c;
}

int graph_sort_bytes(const gzb_engine *e, const GraphCaps &c, int hit_bits, int mw_bits,
                     size_t *bytes) {
  size_t a = 0, b = 0, d = 0, f = 0, g = 0;
  cub::DoubleBuffer<uint32_t> k32(nullptr, nullptr), v32(nullptr, nullptr);
  GZB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, g, k32, v32, (int64_t)c.ext, 0, 16));
  cub::DoubleBuffer<uint64_t> k1(nullptr, nullptr);
  GZB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, a, k1, (int64_t)c.hits, 0, hit_bits));
  GZB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, b, k1, (int64_t)c.mwork, 0, mw_bits));
  const uint64_t *u64 = nullptr;
  uint64_t *o64 = nullptr;
  const uint32_t *u32 = nullptr;
  GZB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, d, u64, o64,
                                         (int64_t)(e->L.n_lists + 1)));
  GZB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, f, u32, o64, (int64_t)(e->nq + 1)));
  *bytes = std::max(std::max(std::max(a, b), std::max(d, f)), g);
  return GZB_OK;
}

// every buffer the graph touches, at its capacity (before capture: the
// capture itself must not allocate)
int graph_prepare(gzb_engine *e, const GraphCaps &c, int hit_bits, int mw_bits, bool learned) {
  const uint32_t nq = e->nq;
  GZB_TRY(e->list_bufs[14].ensure(8 * (e->L.n_lists + 1)));
  GZB_TRY(e->ctr.ensure(64));
  // [0..3] counts, [6] overflow, [8..20] report, [24..30] stage stamps
  GZB_TRY(e->plan.ensure(8 * 32));
  GZB_TRY(e->hits.ensure(8 * (c.hits + 1)));
  GZB_TRY(e->hits_alt.ensure(8 * (c.hits + 1)));
  GZB_TRY(e->hits_copy.ensure(8 * (c.hits + 1)));
  GZB_TRY(e->mwork.ensure(8 * (c.mwork + 1)));
  GZB_TRY(e->mwork_alt.ensure(8 * (c.mwork + 1)));
  GZB_TRY(e->begin.ensure(8 * (nq + 1)));
  GZB_TRY(e->kept.ensure(4 * (nq + 1)));
  GZB_TRY(e->surv_off.ensure(8 * (nq + 1)));
  GZB_TRY(e->slots.ensure(8 * (e->q_len + nq + 1)));
  for (DBuf *b : {&e->eq, &e->ed, &e->escore, &e->elen0, &e->elen1, &e->eqid})
    GZB_TRY(b->ensure(4 * (c.ext + 1)));
  GZB_TRY(e->edir.ensure(c.ext + 1));
  GZB_TRY(e->enb.ensure(4 * (c.hits + 1)));
  GZB_TRY(e->heap.ensure(20 * (c.hits + 1)));  // merge keys and heap slots
  if (learned) {  // the cost-model order
    GZB_TRY(e->efeat.ensure(4 * kFeat * (c.ext + 1)));
    for (DBuf *b : {&e->epred, &e->okeys, &e->okeys2, &e->oidx, &e->oidx2})
      GZB_TRY(b->ensure(4 * (c.ext + 1)));
  }
  size_t tb = 0;
  GZB_TRY(graph_sort_bytes(e, c, hit_bits, mw_bits, &tb));
  GZB_TRY(e->tmp.ensure(tb));
  // the gapped stage's spill lists and fallback band pool
  if (e->spill_cap < 2 * c.ext) {
    cudaFree(e->spill);
    e->spill = nullptr;
    e->spill_cap = 0;
    GZB_CUDA(cudaMalloc(&e->spill, 4 * 2 * c.ext));
    e->spill_cap = 2 * c.ext;
  }
  GZB_TRY(ensure_band_pool(&e->band_pool, &e->band_wmask));
  if (!e->report_h) GZB_CUDA(cudaMallocHost(&e->report_h, 8 * kReportWords));
  if (!e->gstream) GZB_CUDA(cudaStreamCreateWithFlags(&e->gstream, cudaStreamNonBlocking));
  if (!e->gev_in) GZB_CUDA(cudaEventCreateWithFlags(&e->gev_in, cudaEventDisableTiming));
  if (!e->gev_out) GZB_CUDA(cudaEventCreateWithFlags(&e->gev_out, cudaEventDisableTiming));
  return GZB_OK;
}

// the presearch body recorded into the graph
int graph_body(gzb_engine *e, int schedule, const GappedTile &tile, bool learned,
               const GraphCaps &c, int qbits, int dbits, int nqbits, cudaStream_t s,
               uint64_t *launches_out) {
  uint64_t launches = 0;
  DevLists &L = e->L;
  const DevIndex &X = e->X;
  const uint32_t nq = e->nq;
  uint64_t *plan = e->plan.as<uint64_t>();
  uint32_t *overflow = reinterpret_cast<uint32_t *>(plan + 6);
  unsigned long long *ctr = e->ctr.as<unsigned long long>();
  stamp_kernel<<<1, 1, 0, s>>>(plan + 24 + 0);
  GZB_CUDA(cudaMemsetAsync(plan, 0, 64, s));
  GZB_CUDA(cudaMemsetAsync(ctr, 0, 64, s));
  // list lookup; the unit count stays on the device
  if (L.n_lists) {
    uint64_t *unit_counts = e->list_bufs[14].as<uint64_t>();
    list_lookup_kernel<<<grid1(L.n_lists, 256), 256, 0, s>>>(L, X, e->params.clustering,
                                                              unit_counts);
    GZB_CUDA(cudaGetLastError());
    ++launches;
    GZB_CUDA(cudaMemsetAsync(unit_counts + L.n_lists, 0, 8, s));
    GZB_TRY(exclusive_sum(e, unit_counts, L.unit_offsets, L.n_lists + 1, s));
  }
  stamp_kernel<<<1, 1, 0, s>>>(plan + 24 + 1);
  // seed search, distance and ungapped extension
  SeedArgs a;
  a.p = e->dp;
  a.L = L;
  a.X = X;
  a.q = e->q_buf.as<uint8_t>() + kPad;
  a.db = e->db_buf.as<uint8_t>() + kPad;
  a.q_offsets = e->q_offsets.as<uint32_t>();
  a.cutoffs = e->q_cut.as<int32_t>();
  a.triggers = e->q_trig.as<int32_t>();
  a.matrix32 = e->matrix32.as<int32_t>();
  a.clustering = e->params.clustering;
  a.dbits = dbits;
  a.qbits = qbits;
  a.hits = e->hits.as<uint64_t>();
  a.hit_count = ctr + 4;
  a.hit_cap = c.hits;
  a.mwork = e->mwork.as<uint2>();
  a.mwork_count = ctr + 5;
  a.mwork_cap = c.mwork;
  a.ctr = ctr;
  a.units_dev = L.n_lists ? L.unit_offsets + L.n_lists : nullptr;
  if (L.n_lists) {
    if (tile.seed_walker == GZB_SEED_WALKER_DEALT)
      seed_dealt_kernel<<<148 * 16, kSeedBlock, 0, s>>>(a);
    else
      seed_kernel<<<148 * 16, kSeedBlock, 0, s>>>(a);
    GZB_CUDA(cudaGetLastError());
    ++launches;
  }
  // member work in cluster-major order, then the member seeds
  clamp_count_kernel<<<1, 1, 0, s>>>(ctr + 5, c.mwork, plan + 0, overflow, 1u);
  pad_keys_kernel<<<148 * 4, 256, 0, s>>>(reinterpret_cast<uint64_t *>(a.mwork), plan + 0,
                                          c.mwork);
  GZB_CUDA(cudaGetLastError());
  launches += 2;
  uint64_t *sorted_mw = nullptr;
  GZB_TRY(sort_keys_u64(e, reinterpret_cast<uint64_t *>(a.mwork), e->mwork_alt.as<uint64_t>(),
                        c.mwork, bits_for(X.n_reps + 1), s, &sorted_mw));
  ++launches;
  member_kernel<<<148 * 16, kSeedBlock, 0, s>>>(a, reinterpret_cast<const uint2 *>(sorted_mw),
                                                c.mwork, plan + 0);
  GZB_CUDA(cudaGetLastError());
  ++launches;
  stamp_kernel<<<1, 1, 0, s>>>(plan + 24 + 6);
  // hits sorted by (query, database position, query position)
  clamp_count_kernel<<<1, 1, 0, s>>>(ctr + 4, c.hits, plan + 1, overflow, 2u);
  pad_keys_kernel<<<148 * 4, 256, 0, s>>>(e->hits.as<uint64_t>(), plan + 1, c.hits);
  GZB_CUDA(cudaGetLastError());
  launches += 2;
  uint64_t *hits = nullptr;
  GZB_TRY(sort_keys_u64(e, e->hits.as<uint64_t>(), e->hits_alt.as<uint64_t>(), c.hits,
                        qbits + dbits + nqbits, s, &hits));
  ++launches;
  GZB_CUDA(cudaMemcpyAsync(e->hits_copy.p, hits, 8 * c.hits, cudaMemcpyDeviceToDevice, s));
  stamp_kernel<<<1, 1, 0, s>>>(plan + 24 + 2);
  // chain filter
  uint64_t *begin = e->begin.as<uint64_t>();
  uint32_t *kept = e->kept.as<uint32_t>();
  uint64_t *surv_off = e->surv_off.as<uint64_t>();
  hit_segments_kernel<<<grid1(nq + 1, 256), 256, 0, s>>>(hits, c.hits, nq, qbits + dbits, begin,
                                                          plan + 1);
  GZB_CUDA(cudaGetLastError());
  ++launches;
  GZB_TRY(launch_chain(e, nq, hits, begin, qbits, dbits, kept, s));
  GZB_CUDA(cudaGetLastError());
  ++launches;
  GZB_CUDA(cudaMemsetAsync(kept + nq, 0, 4, s));
  GZB_TRY(exclusive_sum(e, kept, surv_off, nq + 1, s));
  ext_count_kernel<<<1, 1, 0, s>>>(surv_off, nq, plan);
  GZB_CUDA(cudaGetLastError());
  launches += 2;
  stamp_kernel<<<1, 1, 0, s>>>(plan + 24 + 3);
  // gapped extension of both sides, in hit order
  build_ext_kernel<<<grid1((uint64_t)nq * 32, 256), 256, 0, s>>>(
      hits, begin, kept, surv_off, nq, e->q_offsets.as<uint32_t>(),
      e->q_lengths.as<uint32_t>(), e->db_offsets.as<uint32_t>(), e->nseq, (uint32_t)e->db_len,
      qbits, dbits, c.hits, e->eq.as<uint32_t>(), e->ed.as<uint32_t>(), e->edir.as<uint8_t>(),
      e->elen0.as<uint32_t>(), e->elen1.as<uint32_t>(), e->eqid.as<uint32_t>(),
      e->enb.as<uint32_t>(), plan + 2, e->q_prev.as<uint32_t>(), e->q_next.as<uint32_t>(),
      learned ? 1 : 0);
  GZB_CUDA(cudaGetLastError());
  ++launches;
  GZB_CUDA(cudaMemsetAsync(e->gcells, 0, 8, s));
  GappedJob job;
  job.query = e->q_buf.as<uint8_t>() + kPad;
  job.db = e->db_buf.as<uint8_t>() + kPad;
  job.delim = e->params.delimiter;
  job.gap_open = e->params.gap_open;
  job.gap_ext = e->params.gap_extension;
  job.cutoff = e->params.gapped_cutoff;
  GappedTile t = tile;
  if (schedule == GZB_SCHEDULE_PLAIN) t.kernel = GZB_GAPPED_KERNEL_STATIC;
  const uint32_t *order = nullptr;
  if (learned) {
    // longest predicted first: features, the cost model, keys, one sort
    ext_features_kernel<<<grid1(c.hits, 256), 256, 0, s>>>(
        job.query, job.db, job.delim, e->matrix32.as<int32_t>(), e->q_cut.as<int32_t>(),
        c.hits, e->eq.as<uint32_t>(), e->ed.as<uint32_t>(), e->elen0.as<uint32_t>(),
        e->elen1.as<uint32_t>(), e->eqid.as<uint32_t>(), e->enb.as<uint32_t>(),
        e->efeat.as<float>(), plan + 2);
    GZB_CUDA(cudaGetLastError());
    GZB_TRY(cost_predict(e->model_d.as<float>(), e->efeat.as<float>(), (uint32_t)c.ext,
                         e->epred.as<float>(), s, plan + 3));
    cost_keys_kernel<<<grid1(c.ext, 256), 256, 0, s>>>(e->epred.as<float>(), nullptr, c.ext,
                                                       e->okeys.as<uint32_t>(),
                                                       e->oidx.as<uint32_t>(), plan + 3, c.ext);
    GZB_CUDA(cudaGetLastError());
    cub::DoubleBuffer<uint32_t> kb(e->okeys.as<uint32_t>(), e->okeys2.as<uint32_t>());
    cub::DoubleBuffer<uint32_t> vb(e->oidx.as<uint32_t>(), e->oidx2.as<uint32_t>());
    size_t tb = e->tmp.bytes;
    GZB_CUDA(cub::DeviceRadixSort::SortPairs(e->tmp.p, tb, kb, vb, (int64_t)c.ext, 0, 16, s));
    order = vb.Current();
    launches += 4;
  }
  GZB_TRY(run_gapped(t, job, e->matrix32.as<int32_t>(), 32, 32, c.ext, order, 0,
                     e->edir.as<uint8_t>(), e->eq.as<uint32_t>(), e->ed.as<uint32_t>(),
                     e->escore.as<int32_t>(), &e->spill, &e->spill_cap, e->gcounters,
                     e->gcells, nullptr, &e->band_pool, &e->band_wmask, s, nullptr, plan + 3));
  launches += 3;
  stamp_kernel<<<1, 1, 0, s>>>(plan + 24 + 4);
  // top-b merge (nothing when a count overflowed)
  merge_kernel<<<grid1((uint64_t)nq * 32, 128), 128, 0, s>>>(
      nq, hits, begin, kept, surv_off, c.hits, e->eq.as<uint32_t>(), e->ed.as<uint32_t>(),
      e->escore.as<int32_t>(), e->q_offsets.as<uint32_t>(), qbits, dbits,
      e->db_offsets.as<uint32_t>(), e->nseq, (uint32_t)e->db_len, e->chunk_id,
      e->params.max_number_results, e->params.max_number_one_subject_results,
      e->heap.as<ulonglong2>(),
      reinterpret_cast<uint32_t *>(e->heap.as<ulonglong2>() + c.hits + 1),
      e->results.as<gzb_result>(), e->counts.as<uint32_t>(), plan + 2, overflow);
  GZB_CUDA(cudaGetLastError());
  ++launches;
  stamp_kernel<<<1, 1, 0, s>>>(plan + 24 + 5);
  report_kernel<<<1, 1, 0, s>>>(ctr, plan, e->gcells, e->gcounters, plan + 8);
  GZB_CUDA(cudaGetLastError());
  ++launches;
  GZB_CUDA(cudaMemcpyAsync(e->report_h, plan + 8, 8 * kReportWords, cudaMemcpyDeviceToHost, s));
  *launches_out = launches + 7;  // and the seven stage stamps
  return GZB_OK;
}

uint64_t fnv_mix(uint64_t h, const void *p, size_t n) {
  const uint8_t *b = (const uint8_t *)p;
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}

// what a captured graph depends on: every buffer it touches (address and
// size), the chunk, the queries, the schedule, the tile and the capacities
uint64_t graph_key(const gzb_engine *e, int schedule, const GappedTile &tile, bool learned,
                   const GraphCaps &c) {
  uint64_t h = 1469598103934665603ull;
  const DBuf *bufs[] = {&e->db_buf, &e->db_offsets, &e->q_buf, &e->q_offsets, &e->q_lengths,
                        &e->q_cut, &e->q_trig, &e->matrix32, &e->results, &e->counts,
                        &e->tmp, &e->hits, &e->hits_alt, &e->hits_copy, &e->mwork,
                        &e->mwork_alt, &e->begin, &e->kept, &e->surv_off, &e->slots, &e->eq,
                        &e->ed, &e->edir, &e->escore, &e->elen0, &e->elen1, &e->eqid, &e->enb,
                        &e->heap, &e->ctr, &e->plan, &e->list_bufs[14],
                        &e->efeat, &e->epred, &e->okeys, &e->okeys2, &e->oidx, &e->oidx2,
                        &e->model_d, &e->q_prev, &e->q_next};
  for (const DBuf *b : bufs) {
    h = fnv_mix(h, &b->p, sizeof(b->p));
    h = fnv_mix(h, &b->bytes, sizeof(b->bytes));
  }
  h = fnv_mix(h, &e->X, sizeof(e->X));
  h = fnv_mix(h, &e->L, sizeof(e->L));
  h = fnv_mix(h, &e->dp, sizeof(e->dp));
  h = fnv_mix(h, &e->params, sizeof(e->params));
  const uint64_t v[] = {e->db_len, e->nseq, (uint64_t)(int64_t)e->chunk_id, e->nq, e->q_len,
                        e->max_qlen, (uint64_t)schedule, (uint64_t)tile.kernel,
                        (uint64_t)tile.book_threshold, (uint64_t)tile.order,
                        (uint64_t)tile.seed_walker, (uint64_t)tile.band_width, c.hits, c.mwork,
                        (uint64_t)(uintptr_t)e->spill, e->spill_cap,
                        (uint64_t)(uintptr_t)e->band_pool, (uint64_t)(uintptr_t)e->gcounters,
                        (uint64_t)(uintptr_t)e->gcells, (uint64_t)(uintptr_t)e->report_h,
                        (uint64_t)learned};
  return fnv_mix(h, v, sizeof(v));
}

void drop_graphs(gzb_engine *e) {
  for (auto &g : e->graphs) cudaGraphExecDestroy(g.exec);
  e->graphs.clear();
}

int presearch_graph(gzb_engine *e, int schedule, const GappedTile &tile, bool learned,
                    cudaStream_t user) {
  const uint32_t nq = e->nq;
  const int qbits = bits_for(e->max_qlen);
  const int dbits = bits_for(e->db_len + 1);
  const int nqbits = bits_for(nq);
  GZB_CHECK(qbits + dbits + nqbits <= 64, GZB_ERR_OVERFLOW,
            "hit key needs %d bits (queries %u, chunk %llu, longest query %u)",
            qbits + dbits + nqbits, nq, (unsigned long long)e->db_len, e->max_qlen);
  const GraphCaps c = graph_caps(e);
  GZB_CHECK(c.ext < (1ull << 32), GZB_ERR_OVERFLOW, "graph mode: extension capacity above 2^32");
  GZB_TRY(graph_prepare(e, c, qbits + dbits + nqbits, bits_for(e->X.n_reps + 1), learned));
  const uint64_t key = graph_key(e, schedule, tile, learned, c);
  gzb_engine::GraphEntry *g = nullptr;
  for (auto &x : e->graphs)
    if (x.key == key) g = &x;
  cudaStream_t s = e->gstream;
  if (!g) {
    if ((int)e->graphs.size() >= kGraphCache) {  // drop the least recently used
      size_t oldest = 0;
      for (size_t i = 1; i < e->graphs.size(); ++i)
        if (e->graphs[i].used < e->graphs[oldest].used) oldest = i;
      cudaGraphExecDestroy(e->graphs[oldest].exec);
      e->graphs.erase(e->graphs.begin() + oldest);
    }
    GZB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    uint64_t launches = 0;
    const int rc = graph_body(e, schedule, tile, learned, c, qbits, dbits, nqbits, s, &launches);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (rc != GZB_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    GZB_CUDA(ce);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    GZB_CUDA(ie);
    e->graphs.push_back(gzb_engine::GraphEntry{key, exec, launches, 0});
    g = &e->graphs.back();
    ++e->graph_captures;
  }
  g->used = ++e->graph_clock;
  e->qbits = qbits;
  e->dbits = dbits;
  GZB_CUDA(cudaEventRecord(e->gev_in, user));
  GZB_CUDA(cudaStreamWaitEvent(s, e->gev_in, 0));
  GZB_CUDA(cudaGraphLaunch(g->exec, s));
  GZB_CUDA(cudaEventRecord(e->gev_out, s));
  GZB_CUDA(cudaStreamWaitEvent(user, e->gev_out, 0));
  GZB_CUDA(cudaStreamSynchronize(s));
  ++e->graph_replays;
  const uint64_t *r = e->report_h;
  if (r[11] != 0) {
    // a count above its capacity: nothing was merged; grow and redo eagerly
    ++e->graph_fallbacks;
    e->hit_cap = std::max<uint64_t>(e->hit_cap, r[4] + r[4] / 8 + 1024);
    e->mwork_cap = std::max<uint64_t>(e->mwork_cap, r[5] + r[5] / 8 + 1024);
    drop_graphs(e);
    return presearch_impl(e, schedule, user);
  }
  GZB_CHECK(r[10] == 0, GZB_ERR_OVERFLOW,
            "%llu gapped extensions need a band wider than the fallback's",
            (unsigned long long)r[10]);
  e->counters.distance_seeds = r[0];
  e->counters.ungapped_seeds = r[1];
  e->counters.ungapped_steps = r[2];
  e->counters.ungapped_hits = r[12];
  e->counters.chained_hits = r[6];
  e->counters.gapped_extensions = 2 * r[6];
  e->counters.gapped_cells = r[7];
  e->counters.gapped_fallbacks = r[8];
  e->counters.kernel_launches = g->launches;
  e->last_mae = -1.0f;
  e->last_mae_n = 0;
  e->pred_n = learned ? 2 * r[6] : 0;
  e->prev_cells_n = 0;
  // stage stamps at the points where the eager path records ev[0..6]
  const uint64_t *stamp = r + 16;
  auto ms = [&](int a, int b) { return (float)((double)(int64_t)(stamp[b] - stamp[a]) * 1e-6); };
  for (int i = 0; i < 5; ++i) e->stage_ms[i] = ms(i, i + 1);
  e->stage_ms[5] = ms(0, 5);
  e->stage_ms[6] = ms(1, 6);
  return GZB_OK;
}

}  // namespace

extern "C" int gzb_engine_set_graph(gzb_engine *e, int enable) {
  GZB_TRY(check_engine(e));
  e->graph = enable != 0;
  if (!e->graph) drop_graphs(e);
  return GZB_OK;
}

extern "C" int gzb_engine_reserve(gzb_engine *e, uint64_t hits, uint64_t member_work) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(hits >= 1 && member_work >= 1 && hits < (1ull << 40) && member_work < (1ull << 40),
            GZB_ERR_INVALID, "capacities must be in 1 .. 2^40");
  e->hit_cap = hits;
  e->mwork_cap = member_work;
  drop_graphs(e);
  return GZB_OK;
}

extern "C" int gzb_engine_get_graph_stats(gzb_engine *e, uint64_t *captures, uint64_t *replays,
                                          uint64_t *fallbacks) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(captures && replays && fallbacks, GZB_ERR_INVALID, "null argument");
  *captures = e->graph_captures;
  *replays = e->graph_replays;
  *fallbacks = e->graph_fallbacks;
  return GZB_OK;
}

extern "C" int gzb_engine_presearch(gzb_engine *e, int schedule, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_db && e->have_queries, GZB_ERR_INVALID,
            "set_database and set_queries first");
  GZB_CHECK(schedule == GZB_SCHEDULE_PLAIN || schedule == GZB_SCHEDULE_BATCHED ||
                schedule == GZB_SCHEDULE_ORACLE,
            GZB_ERR_INVALID, "unknown schedule %d", schedule);
  GZB_CHECK(e->params.max_number_one_subject_results <= 4, GZB_ERR_INVALID,
            "max_number_one_subject_results above 4 is not supported");
  if (e->graph && schedule != GZB_SCHEDULE_ORACLE && !e->logging) {
    // graph mode covers hit order; a cost-model order runs eagerly
    GappedTile tile = g_tile;
    for (int w = 0; w < kTileParameters; ++w)
      if (e->tile[schedule][w] >= 0) *tile_field(tile, w) = e->tile[schedule][w];
    const bool learned =
        schedule == GZB_SCHEDULE_BATCHED && e->have_model && tile.order == GZB_ORDER_MODEL;
    return presearch_graph(e, schedule, tile, learned, (cudaStream_t)stream);
  }
  return presearch_impl(e, schedule, (cudaStream_t)stream);
}

extern "C" int gzb_engine_get_results(gzb_engine *e, uint32_t *counts, gzb_result *results,
                                      void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_queries && counts && results, GZB_ERR_INVALID, "no results");
  cudaStream_t s = (cudaStream_t)stream;
  GZB_CUDA(cudaMemcpyAsync(counts, e->counts.p, 4 * (uint64_t)e->nq, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaMemcpyAsync(results, e->results.p,
                           sizeof(gzb_result) * (uint64_t)e->nq * e->params.max_number_results,
                           cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  return GZB_OK;
}

namespace {
// exclusive scan of n + 1 entries (the last one zeroed first); returns the total
int scan_total(gzb_engine *e, DBuf &in, DBuf &out, uint64_t n, cudaStream_t s,
               uint64_t *total) {
  GZB_TRY(out.ensure(8 * (n + 1)));
  GZB_CUDA(cudaMemsetAsync(in.as<uint64_t>() + n, 0, 8, s));
  GZB_TRY(exclusive_sum(e, in.as<uint64_t>(), out.as<uint64_t>(), n + 1, s));
  GZB_CUDA(cudaMemcpyAsync(total, out.as<uint64_t>() + n, 8, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  return GZB_OK;
}

// the two scans of the flagged sides' storage sizes with one host wait
int scan_totals2(gzb_engine *e, uint64_t n, cudaStream_t s, uint64_t *ops_total,
                 uint64_t *rows_total) {
  DBuf *in[2] = {&e->tb_ops_bytes, &e->tb_rows};
  DBuf *out[2] = {&e->tb_ops_off, &e->tb_rows_off};
  uint64_t *total[2] = {ops_total, rows_total};
  for (int k = 0; k < 2; ++k) {
    GZB_TRY(out[k]->ensure(8 * (n + 1)));
    GZB_CUDA(cudaMemsetAsync(in[k]->as<uint64_t>() + n, 0, 8, s));
    GZB_TRY(exclusive_sum(e, in[k]->as<uint64_t>(), out[k]->as<uint64_t>(), n + 1, s));
    GZB_CUDA(cudaMemcpyAsync(total[k], out[k]->as<uint64_t>() + n, 8, cudaMemcpyDeviceToHost,
                             s));
  }
  GZB_CUDA(cudaStreamSynchronize(s));
  return GZB_OK;
}
}  // namespace

extern "C" int gzb_engine_build_alignments(gzb_engine *e, uint32_t *counts,
                                           gzb_alignment *alignments, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_db && e->have_queries && counts && alignments, GZB_ERR_INVALID,
            "build alignments needs the chunk, the queries and output arrays");
  cudaStream_t s = (cudaStream_t)stream;
  const int b = e->params.max_number_results;
  const uint64_t n_slots = (uint64_t)e->nq * b, n_sides = 2 * n_slots;
  TbArgs a;
  a.query = e->q_buf.as<uint8_t>() + kPad;
  a.db = e->db_buf.as<uint8_t>() + kPad;
  a.matrix32 = e->matrix32.as<int32_t>();
  a.q_offsets = e->q_offsets.as<uint32_t>();
  a.q_lengths = e->q_lengths.as<uint32_t>();
  a.results = e->results.as<gzb_result>();
  a.counts = e->counts.as<uint32_t>();
  a.nq = e->nq;
  a.max_results = b;
  a.chunk_id = e->chunk_id;
  a.delim = e->params.delimiter;
  a.gap_open = e->params.gap_open;
  a.gap_ext = e->params.gap_extension;
  // the build results step's own X-drop (src/aligner_gpu.cpp:254-256)
  a.cutoff = e->params.result_gapped_cutoff;
  GZB_TRY(e->tb_ops_bytes.ensure(8 * (n_sides + 1)));
  GZB_TRY(e->tb_rows.ensure(8 * (n_sides + 1)));
  GZB_TRY(e->tb_redo.ensure(n_sides + 1));
  GZB_TRY(e->tb_score.ensure(4 * (n_sides + 1)));
  GZB_TRY(e->tb_p0.ensure(4 * (n_sides + 1)));
  GZB_TRY(e->tb_p1.ensure(4 * (n_sides + 1)));
  GZB_TRY(e->tb_stats.ensure(sizeof(TbStats) * (n_sides + 1)));
  GZB_TRY(e->tb_out.ensure(sizeof(gzb_alignment) * (n_slots + 1)));
  // one DP pass by warps (each gathering sides' ops and rows in its own
  // scratch, then walking them); the sides a warp cannot run go to the
  // thread kernels
  int sms = 148, per_sm = 1;
  GZB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device));
  GZB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tb_side_warp_kernel,
                                                         kTbWarpBlock, 0));
  const uint64_t want = (n_sides + kTbWarpBlock / 32 - 1) / (kTbWarpBlock / 32);
  const uint64_t blocks = std::max<uint64_t>(
      1, std::min<uint64_t>(want, (uint64_t)sms * std::max(per_sm, 1)));
  GZB_TRY(e->tb_scratch.ensure(blocks * (kTbWarpBlock / 32) * kTbScratchBytes));
  tb_side_warp_kernel<<<(unsigned)blocks, kTbWarpBlock, 0, s>>>(
      a, n_sides, e->tb_scratch.as<uint8_t>(), e->tb_score.as<int32_t>(),
      e->tb_p0.as<int32_t>(), e->tb_p1.as<int32_t>(), e->tb_stats.as<TbStats>(),
      e->tb_ops_bytes.as<uint64_t>(), e->tb_rows.as<uint64_t>(), e->tb_redo.as<uint8_t>());
  GZB_CUDA(cudaGetLastError());
  // the flagged sides' bands (global memory) and storage sizes
  GZB_TRY(e->tb_cols.ensure(8 * (n_sides + 1)));
  tb_band_kernel<<<grid1(n_sides, 256), 256, 0, s>>>(a, n_sides, e->tb_redo.as<uint8_t>(),
                                                     e->tb_cols.as<uint64_t>());
  GZB_CUDA(cudaGetLastError());
  uint64_t band_total = 0;
  GZB_TRY(scan_total(e, e->tb_cols, e->tb_band_off, n_sides, s, &band_total));
  GZB_TRY(e->tb_band.ensure(sizeof(int2) * (band_total + 1)));
  tb_count_kernel<<<grid1(n_sides, 128), 128, 0, s>>>(
      a, n_sides, e->tb_band_off.as<uint64_t>(), e->tb_band.as<int2>(),
      e->tb_ops_bytes.as<uint64_t>(), e->tb_rows.as<uint64_t>(), e->tb_redo.as<uint8_t>());
  GZB_CUDA(cudaGetLastError());
  uint64_t ops_total = 0, rows_total = 0;
  GZB_TRY(scan_totals2(e, n_sides, s, &ops_total, &rows_total));
  GZB_TRY(e->tb_ops.ensure(ops_total + 1));
  GZB_TRY(e->tb_row_meta.ensure(8 * (rows_total + 1)));
  // a cell the thread DP prunes keeps op 0, as in a fresh GappedExtender
  GZB_CUDA(cudaMemsetAsync(e->tb_ops.p, 0, ops_total + 1, s));
  tb_walk_kernel<<<grid1(n_sides, 128), 128, 0, s>>>(
      a, n_sides, e->tb_band_off.as<uint64_t>(), e->tb_band.as<int2>(),
      e->tb_ops_off.as<uint64_t>(), e->tb_ops.as<uint8_t>(), e->tb_rows_off.as<uint64_t>(),
      e->tb_row_meta.as<uint32_t>(), e->tb_score.as<int32_t>(), e->tb_p0.as<int32_t>(),
      e->tb_p1.as<int32_t>(), e->tb_stats.as<TbStats>(), e->tb_redo.as<uint8_t>());
  GZB_CUDA(cudaGetLastError());
  tb_combine_kernel<<<grid1(n_slots, 128), 128, 0, s>>>(
      a, n_slots, e->tb_score.as<int32_t>(), e->tb_p0.as<int32_t>(), e->tb_p1.as<int32_t>(),
      e->tb_stats.as<TbStats>(), e->tb_out.as<gzb_alignment>());
  GZB_CUDA(cudaGetLastError());
  GZB_CUDA(cudaMemcpyAsync(counts, e->counts.p, 4 * (uint64_t)e->nq, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaMemcpyAsync(alignments, e->tb_out.p, sizeof(gzb_alignment) * n_slots,
                           cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  return GZB_OK;
}

extern "C" int gzb_engine_get_counters(gzb_engine *e, gzb_counters *out) {
  GZB_CHECK(e && out, GZB_ERR_INVALID, "null argument");
  *out = e->counters;
  return GZB_OK;
}

extern "C" int gzb_engine_get_stage_ms(gzb_engine *e, float *ms7) {
  GZB_CHECK(e && ms7, GZB_ERR_INVALID, "null argument");
  for (int i = 0; i < 7; ++i) ms7[i] = e->stage_ms[i];
  return GZB_OK;
}

extern "C" int gzb_engine_get_hits(gzb_engine *e, uint32_t *qid, uint32_t *qpos, uint32_t *dpos,
                                   uint64_t capacity, uint64_t *count, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(count, GZB_ERR_INVALID, "null count");
  const uint64_t n = e->counters.ungapped_hits;
  *count = n;
  const uint64_t c = std::min(n, capacity);
  if (c == 0 || !qid || !qpos || !dpos) return GZB_OK;
  std::vector<uint64_t> keys(c);
  cudaStream_t s = (cudaStream_t)stream;
  GZB_CUDA(cudaMemcpyAsync(keys.data(), e->hits_copy.p, 8 * c, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  const uint64_t qmask = (1ull << e->qbits) - 1, dmask = (1ull << e->dbits) - 1;
  for (uint64_t i = 0; i < c; ++i) {
    qpos[i] = (uint32_t)(keys[i] & qmask);
    dpos[i] = (uint32_t)((keys[i] >> e->qbits) & dmask);
    qid[i] = (uint32_t)(keys[i] >> (e->qbits + e->dbits));
  }
  return GZB_OK;
}

__global__ void entry_positions_kernel(const uint32_t *qid, const uint32_t *cpos, uint64_t n,
                                       const uint32_t *q_offsets, uint32_t *out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = cpos[i] - q_offsets[qid[i]];
}

extern "C" int gzb_engine_get_list_array(gzb_engine *e, int which, uint32_t *out,
                                         uint64_t capacity, uint64_t *count, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_queries && count, GZB_ERR_INVALID, "no queries");
  const DevLists &L = e->L;
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t *src = nullptr;
  uint64_t n = 0;
  switch (which) {
    case 0: src = L.hash; n = L.n_lists; break;
    case 1: src = L.offsets; n = L.n_lists + 1; break;
    case 2: src = L.nchk; n = L.n_lists; break;
    case 3: src = L.entry_qid; n = L.n_entries; break;
    case 4: {
      n = L.n_entries;
      GZB_TRY(e->list_bufs[15].ensure(4 * (n + 1)));
      if (n) {
        entry_positions_kernel<<<grid1(n, 256), 256, 0, s>>>(L.entry_qid, L.entry_cpos, n,
                                                             e->q_offsets.as<uint32_t>(),
                                                             e->list_bufs[15].as<uint32_t>());
        GZB_CUDA(cudaGetLastError());
      }
      src = e->list_bufs[15].as<uint32_t>();
      break;
    }
    default: return set_error(GZB_ERR_INVALID, "unknown list array %d", which);
  }
  *count = n;
  if (out && n) {
    const uint64_t c = std::min(n, capacity);
    GZB_CUDA(cudaMemcpyAsync(out, src, 4 * c, cudaMemcpyDeviceToHost, s));
    GZB_CUDA(cudaStreamSynchronize(s));
  }
  return GZB_OK;
}

extern "C" int gzb_engine_get_index_array(gzb_engine *e, int which, uint32_t *out,
                                          uint64_t capacity, uint64_t *count, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(e->have_db && count, GZB_ERR_INVALID, "no database");
  const DevIndex &X = e->X;
  const uint32_t *src = nullptr;
  uint64_t n = 0;
  switch (which) {
    case 0: src = X.nc_keys; n = X.n_nc_keys; break;
    case 1: src = X.nc_offsets; n = X.n_nc_keys + 1; break;
    case 2: src = X.nc_values; n = X.n_nc_values; break;
    case 3: src = X.rep_keys; n = X.n_rep_keys; break;
    case 4: src = X.rep_offsets; n = X.n_rep_keys + 1; break;
    case 5: src = X.rep_cluster_ids; n = X.n_reps; break;
    case 6: src = X.rep_positions; n = X.n_reps; break;
    case 7: src = X.member_offsets; n = X.n_reps + 1; break;
    case 8: src = X.member_positions; n = X.n_members; break;
    default: return set_error(GZB_ERR_INVALID, "unknown index array %d", which);
  }
  *count = n;
  if (out && n) {
    const uint64_t c = std::min(n, capacity);
    cudaStream_t s = (cudaStream_t)stream;
    GZB_CUDA(cudaMemcpyAsync(out, src, 4 * c, cudaMemcpyDeviceToHost, s));
    GZB_CUDA(cudaStreamSynchronize(s));
  }
  return GZB_OK;
}

// ---- cost model and logging ----------------------------------------------

extern "C" int gzb_engine_set_logging(gzb_engine *e, int enable, uint64_t capacity) {
  GZB_TRY(check_engine(e));
  e->logging = enable != 0;
  if (e->logging) {
    GZB_CHECK(capacity > 0, GZB_ERR_INVALID, "zero log capacity");
    GZB_TRY(e->log_x.ensure(4 * kFeat * capacity));
    GZB_TRY(e->log_y.ensure(4 * capacity));
    GZB_TRY(e->log_ctr.ensure(8));
    GZB_CUDA(cudaMemset(e->log_ctr.p, 0, 8));
    e->log_cap = capacity;
  }
  return GZB_OK;
}

extern "C" int gzb_engine_get_log(gzb_engine *e, float *features, float *log_cells,
                                  uint64_t capacity, uint64_t *count) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(count, GZB_ERR_INVALID, "null count");
  uint64_t n = 0;
  if (e->log_ctr.p) GZB_CUDA(cudaMemcpy(&n, e->log_ctr.p, 8, cudaMemcpyDeviceToHost));
  n = std::min(n, e->log_cap);
  *count = n;
  const uint64_t c = std::min(n, capacity);
  if (c && features) GZB_CUDA(cudaMemcpy(features, e->log_x.p, 4 * kFeat * c, cudaMemcpyDeviceToHost));
  if (c && log_cells) GZB_CUDA(cudaMemcpy(log_cells, e->log_y.p, 4 * c, cudaMemcpyDeviceToHost));
  return GZB_OK;
}

extern "C" int gzb_engine_set_cost_model(gzb_engine *e, const float *params) {
  GZB_TRY(check_engine(e));
  if (!params) {
    e->have_model = false;
    return GZB_OK;
  }
  GZB_TRY(e->model_d.ensure(4 * kParams));
  GZB_CUDA(cudaMemcpy(e->model_d.p, params, 4 * kParams, cudaMemcpyHostToDevice));
  e->have_model = true;
  return GZB_OK;
}

extern "C" int gzb_engine_train_cost_model(gzb_engine *e, int epochs, int batch, float lr,
                                           uint64_t seed, float *params, float *final_loss) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(params, GZB_ERR_INVALID, "null params");
  uint64_t n = 0;
  if (e->log_ctr.p) GZB_CUDA(cudaMemcpy(&n, e->log_ctr.p, 8, cudaMemcpyDeviceToHost));
  n = std::min(n, e->log_cap);
  GZB_CHECK(n > 0, GZB_ERR_INVALID, "no logged extensions to train on");
  GZB_CHECK(n < (1ull << 32), GZB_ERR_OVERFLOW, "training set too large");
  GZB_TRY(cost_train(e->log_x.as<float>(), e->log_y.as<float>(), (uint32_t)n, params, epochs,
                     batch, lr, seed, final_loss, 0));
  return gzb_engine_set_cost_model(e, params);
}

extern "C" int gzb_engine_get_schedule_stats(gzb_engine *e, float *mean_abs_log2_error,
                                             uint64_t *count) {
  GZB_CHECK(e && mean_abs_log2_error && count, GZB_ERR_INVALID, "null argument");
  *mean_abs_log2_error = e->last_mae;
  *count = e->last_mae_n;
  return GZB_OK;
}

extern "C" int gzb_engine_get_extension_costs(gzb_engine *e, float *predicted,
                                              uint32_t *cells, uint64_t capacity,
                                              uint64_t *count, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(count, GZB_ERR_INVALID, "null count");
  const uint64_t n = e->prev_cells_n;
  *count = n;
  if (!predicted && !cells) return GZB_OK;
  GZB_CHECK(capacity >= n, GZB_ERR_INVALID, "capacity %llu below %llu extensions",
            (unsigned long long)capacity, (unsigned long long)n);
  GZB_CHECK(!predicted || e->pred_n == n, GZB_ERR_INVALID,
            "the last run made no cost predictions (batched schedule with a model)");
  cudaStream_t s = (cudaStream_t)stream;
  if (n && cells)
    GZB_CUDA(cudaMemcpyAsync(cells, e->prev_cells.p, 4 * n, cudaMemcpyDefault, s));
  if (n && predicted)
    GZB_CUDA(cudaMemcpyAsync(predicted, e->epred.p, 4 * n, cudaMemcpyDefault, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  return GZB_OK;
}

extern "C" int gzb_engine_set_tile(gzb_engine *e, int schedule, int which, int value) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(schedule >= 0 && schedule < 3, GZB_ERR_INVALID, "unknown schedule %d", schedule);
  GZB_TRY(check_tile_value(which, value != -1 ? value : any_tile_value(which)));
  e->tile[schedule][which] = value;
  return GZB_OK;
}

extern "C" int gzb_engine_get_tile(gzb_engine *e, int schedule, int which, int *value) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(value, GZB_ERR_INVALID, "null value");
  GZB_CHECK(schedule >= 0 && schedule < 3, GZB_ERR_INVALID, "unknown schedule %d", schedule);
  GZB_TRY(check_tile_value(which, any_tile_value(which)));
  const int v = e->tile[schedule][which];
  if (v >= 0) *value = v;
  else GZB_TRY(gzb_get_tile_parameter(which, value));
  return GZB_OK;
}

extern "C" int gzb_engine_autotune(gzb_engine *e, int schedule, int which, const int *candidates,
                                   int n, int *best, float *ms, void *stream) {
  GZB_TRY(check_engine(e));
  GZB_CHECK(candidates && n > 0 && best, GZB_ERR_INVALID, "no candidates");
  GZB_CHECK(schedule >= 0 && schedule < 3, GZB_ERR_INVALID, "unknown schedule %d", schedule);
  for (int i = 0; i < n; ++i) GZB_TRY(check_tile_value(which, candidates[i]));
  const int keep = e->tile[schedule][which];
  float best_ms = 1e30f;
  int best_v = candidates[0];
  for (int i = 0; i < n; ++i) {
    e->tile[schedule][which] = candidates[i];
    float t = 0.0f;
    for (int rep = 0; rep < 2; ++rep) {  // the first run warms caches and buffers
      int rc = gzb_engine_reset_results(e, stream);
      if (rc == GZB_OK) rc = gzb_engine_presearch(e, schedule, stream);
      if (rc != GZB_OK) {
        e->tile[schedule][which] = keep;
        return rc;
      }
      // the stage the parameter acts on: seed search or gapped
      t = e->stage_ms[which == GZB_TILE_SEED_WALKER ? 1 : 3];
    }
    if (ms) ms[i] = t;
    if (t < best_ms) {
      best_ms = t;
      best_v = candidates[i];
    }
  }
  e->tile[schedule][which] = best_v;
  GZB_TRY(gzb_engine_reset_results(e, stream));
  *best = best_v;
  return GZB_OK;
}
