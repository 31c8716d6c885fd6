// gzb_noalloc.cu -- gapped one-side extension for callers that cannot
// allocate device memory.
//
// Who needs it: a caller that must not call cudaMalloc itself -- for
// example code embedded in a host runtime that owns every device buffer
// through its own pool, or a latency-critical loop that cannot accept the
// implicit device synchronisation of an allocation.  The regular entry point
// gzb_gapped_extender_extend_one_side_score_only_async allocates its scratch
// (overflow lists, counters, fallback bands) on first use; this one keeps
// that scratch in one file-scope device array instead and allocates
// nothing.  The caller still passes every input and output buffer.
//
// Limits and sharing rules:
//  * at most kNoAllocMaxExtensions extensions per call (larger sizes are
//    rejected with GZB_ERR_OVERFLOW);
//  * the rare extensions that need the serial fallback may use a band of at
//    most kNoAllocBand columns (query remainders up to kNoAllocBand - 2
//    residues); wider ones are reported as GZB_ERR_OVERFLOW after every
//    kernel has run, so on that return the position and score buffers are
//    undefined (the other extensions have already moved their positions in
//    place): a caller that wants to retry must keep its own copy of the
//    input positions;
//  * the array (about 12 MB) is held by every GPU that loads the library
//    until the process exits;
//  * every call shares the array, and it keeps the last call's contents:
//    calls that overlap on the GPU (from several host threads or streams at
//    once) race with each other and must be serialised by the caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) once for that device, so it should come before
//    any stream capture; every call ends by copying a counter to host memory
//    and synchronising `stream`.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "ghostz_b200.h"
#include "gzb_common.h"
#include "gzb_kernels.cuh"

namespace gzb {

// kernels of the regular gapped extender (gzb_operators.cu)
__global__ void gapped_lane_kernel(GappedJob job, const int32_t *__restrict__ matrix,
                                   int number_letters, int stride, size_t n,
                                   const uint32_t *__restrict__ order, int reverse,
                                   const uint8_t *__restrict__ dir, uint32_t *qpos,
                                   uint32_t *dpos, int32_t *scores, uint32_t *spill,
                                   uint32_t *spill_count, unsigned long long *cells_total,
                                   uint32_t *cells_out, const uint64_t *n_dev);
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

namespace {

constexpr size_t kNoAllocMaxExtensions = 1u << 20;
constexpr int kNoAllocSerialThreads = 64;
constexpr int kNoAllocBand = 1 << 13;

// Layout of the scratch array (byte offsets, each 256-byte aligned).
constexpr size_t kOffCounters = 0;                       // 4 x uint32
constexpr size_t kOffCells = 256;                        // 1 x uint64
constexpr size_t kOffSpill = 512;                        // 2 x max uint32
constexpr size_t kOffBands = kOffSpill + 2 * 4 * kNoAllocMaxExtensions;
constexpr size_t kScratchBytes =
    kOffBands + sizeof(int2) * (size_t)kNoAllocSerialThreads * kNoAllocBand;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device with that device current.
int scratch_address(unsigned char **out) {
  int dev = 0;
  GZB_CUDA(cudaGetDevice(&dev));
  GZB_CHECK(dev >= 0 && dev < kMaxDevices, GZB_ERR_INVALID, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    GZB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_ptr[dev] = (unsigned char *)p;
  }
  *out = g_scratch_ptr[dev];
  return GZB_OK;
}

}  // namespace
}  // namespace gzb

using namespace gzb;

extern "C" int gzb_gapped_extend_one_side_score_only_noalloc(
    const uint8_t *d_query_sequence, const uint8_t *d_database_sequence,
    uint8_t sequence_delimiter, const int32_t *d_score_matrix, uint32_t number_letters,
    int gap_open, int gap_extension, int cutoff, size_t size, int reverse,
    uint32_t *d_query_concatenated_positions, uint32_t *d_database_positions,
    int32_t *d_scores, void *stream) {
  GZB_CHECK(d_query_sequence && d_database_sequence && d_score_matrix, GZB_ERR_INVALID,
            "null sequence or matrix");
  GZB_CHECK(number_letters > 0 && number_letters < 32, GZB_ERR_INVALID,
            "number_letters %u out of range", number_letters);
  GZB_CHECK(gap_open >= 0 && gap_extension >= 0, GZB_ERR_INVALID, "negative gap penalty");
  GZB_CHECK(size <= kNoAllocMaxExtensions, GZB_ERR_OVERFLOW,
            "%zu extensions exceed the limit of %zu per call without allocation", size,
            kNoAllocMaxExtensions);
  if (size == 0) return GZB_OK;
  GZB_CHECK(d_query_concatenated_positions && d_database_positions && d_scores,
            GZB_ERR_INVALID, "null position or score buffer");
  unsigned char *scratch = nullptr;
  GZB_TRY(scratch_address(&scratch));
  cudaStream_t s = (cudaStream_t)stream;
  uint32_t *counters = (uint32_t *)(scratch + kOffCounters);
  unsigned long long *cells = (unsigned long long *)(scratch + kOffCells);
  uint32_t *spill1 = (uint32_t *)(scratch + kOffSpill);
  uint32_t *spill2 = spill1 + kNoAllocMaxExtensions;
  int2 *bands = (int2 *)(scratch + kOffBands);
  // the counters start at zero on every call (the array keeps old contents)
  GZB_CUDA(cudaMemsetAsync(scratch, 0, kOffSpill, s));
  GappedJob job;
  job.query = d_query_sequence;
  job.db = d_database_sequence;
  job.delim = sequence_delimiter;
  job.gap_open = gap_open;
  job.gap_ext = gap_extension;
  job.cutoff = cutoff;
  const int stride = (int)number_letters + 1;
  int dev = 0, sms = 0;
  GZB_CUDA(cudaGetDevice(&dev));
  GZB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const size_t blocks = (size + 127) / 128, cap = (size_t)sms * 40;
  gapped_lane_kernel<<<(unsigned)(blocks < cap ? blocks : cap), 128, 0, s>>>(
      job, d_score_matrix, (int)number_letters, stride, size, nullptr, reverse, nullptr,
      d_query_concatenated_positions, d_database_positions, d_scores, spill1, counters, cells,
      nullptr, nullptr);
  GZB_CUDA(cudaGetLastError());
  const uint32_t *serial_list = spill1, *serial_count = counters;
  if (warp_path_exact(cutoff)) {
    gapped_warp_kernel<<<sms * 4, 256, 0, s>>>(job, d_score_matrix, (int)number_letters,
                                                stride, spill1, counters, reverse, nullptr,
                                                d_query_concatenated_positions,
                                                d_database_positions, d_scores, spill2,
                                                counters + 1, cells);
    GZB_CUDA(cudaGetLastError());
    serial_list = spill2;
    serial_count = counters + 1;
  }
  gapped_serial_kernel<<<1, kNoAllocSerialThreads, 0, s>>>(
      job, d_score_matrix, (int)number_letters, stride, serial_list, serial_count, reverse,
      nullptr, d_query_concatenated_positions, d_database_positions, d_scores, bands,
      kNoAllocBand - 1, cells, counters + 2);
  GZB_CUDA(cudaGetLastError());
  uint32_t too_long = 0;
  GZB_CUDA(cudaMemcpyAsync(&too_long, counters + 2, 4, cudaMemcpyDeviceToHost, s));
  GZB_CUDA(cudaStreamSynchronize(s));
  GZB_CHECK(too_long == 0, GZB_ERR_OVERFLOW,
            "%u extensions need a band wider than %d columns", too_long, kNoAllocBand);
  return GZB_OK;
}
