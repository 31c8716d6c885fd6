// reference_device_layer.cu -- the device layer of GHOSTZ-GPU's own GPU
// aligner, implemented over this library.
//
// GHOSTZ-GPU keeps everything that touches the GPU in nine CUDA files
// (CU_SRC of its Makefile): the three operators (src/distance_calculator_gpu.cu,
// src/ungapped_extender_gpu.cu, src/gapped_extender_gpu.cu and their three
// kernel files), the device data holder (src/aligner_gpu_data.cu), the
// per-stream device buffers (src/device_seeds_memory.cu) and the code
// packing (src/packed_alphabet_code.cu).  This file defines the classes the
// first eight define -- DistanceCalculatorGpu, UngappedExtenderGpu,
// GappedExtenderGpu, AlignerGpuData, DeviceSeedsMemory -- against the
// reference's own headers, calling libghostz_b200.so.  Compiled with the
// reference's headers on the include path and linked in place of those
// eight objects (plus -lghostz_b200; the packing file's host functions are
// compiled from the reference as they are), it makes the reference's
// `ghostz-gpu aln -g N` run its
// unchanged host code (AlignerGpu, AlignerGpuPresearchThread,
// SeedSearcherGpu, GpuStreamController / GpuStreamRunner, ...) on this
// library's kernels.
//
// Layout the library needs, kept inside AlignerGpuData: sequences are one
// byte per code with 64 delimiter bytes before and after them (instead of
// 12 five-bit codes per 64-bit word behind 4 words of padding); the pointer
// the holder hands out addresses the first code and is only ever passed to
// the operators.  The score matrix keeps the reference's (n + 1)^2 layout.
// Errors: the reference exits on a CUDA failure (CUDA_CHECK_RETURN,
// src/cuda_common.h:13-19); these definitions do the same with the
// library's message.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <vector>

#include "aligner_gpu_data.h"
#include "device_seeds_memory.h"
#include "distance_calculator_gpu.h"
#include "gapped_extender_gpu.h"
#include "ghostz_b200.h"
#include "ungapped_extender_gpu.h"

namespace {

constexpr size_t kSequencePad = 64;  // delimiter bytes around device sequences

void die(int rc, const char *what) {
  if (rc == GZB_OK) return;
  fprintf(stderr, "libghostz_b200 %s: %s\n", what, gzb_last_error());
  exit(1);
}

// one library handle per reference object (the reference's classes keep
// only raw pointers, so the handle lives beside the object)
template <class H>
class Handles {
 public:
  void add(const void *owner, H *h) {
    std::lock_guard<std::mutex> lock(m_);
    map_[owner] = h;
  }
  H *get(const void *owner) {
    std::lock_guard<std::mutex> lock(m_);
    return map_.at(owner);
  }
  H *take(const void *owner) {
    std::lock_guard<std::mutex> lock(m_);
    H *h = map_.at(owner);
    map_.erase(owner);
    return h;
  }

 private:
  std::mutex m_;
  std::map<const void *, H *> map_;
};

Handles<gzb_distance_calculator> g_distance;
Handles<gzb_ungapped_extender> g_ungapped;
Handles<gzb_gapped_extender> g_gapped;

const uint8_t *bytes(const packed_alphabet_code::PackedAlphabetCode *p) {
  return reinterpret_cast<const uint8_t *>(p);
}

// `length` codes between kSequencePad delimiter bytes (the delimiter is the
// sequence's first code: concatenated sequences start with one), in the
// holder's device vector; returns the address of the first code
packed_alphabet_code::PackedAlphabetCode *upload_codes(
    thrust::device_vector<packed_alphabet_code::PackedAlphabetCode> &buf,
    const AlphabetCoder::Code *codes, size_t length) {
  const size_t total = length + 2 * kSequencePad;
  const size_t words = (total + 7) / 8;
  if (buf.size() < words) buf.resize(words);
  uint8_t *base = reinterpret_cast<uint8_t *>(thrust::raw_pointer_cast(buf.data()));
  const int delimiter = length ? codes[0] : 0;
  if (cudaMemset(base, delimiter, words * 8) != cudaSuccess ||
      cudaMemcpy(base + kSequencePad, codes, length, cudaMemcpyHostToDevice) != cudaSuccess) {
    fprintf(stderr, "AlignerGpuData: sequence upload failed\n");
    exit(1);
  }
  return reinterpret_cast<packed_alphabet_code::PackedAlphabetCode *>(base + kSequencePad);
}

}  // namespace

// ---- AlignerGpuData (src/aligner_gpu_data.h) ------------------------------
AlignerGpuData::AlignerGpuData() : gpu_id_(0) {}

AlignerGpuData::AlignerGpuData(int gpu_id) : gpu_id_(gpu_id) { SetGpuId(gpu_id); }

AlignerGpuData::~AlignerGpuData() {}

void AlignerGpuData::SetGpuId(int gpu_id) {
  gpu_id_ = gpu_id;
  if (cudaSetDevice(gpu_id_) != cudaSuccess) {
    fprintf(stderr, "AlignerGpuData: cudaSetDevice(%d) failed\n", gpu_id_);
    exit(1);
  }
}

int AlignerGpuData::GetGpuId() { return gpu_id_; }

void AlignerGpuData::SetGpuQueryIds(uint32_t *query_ids, size_t length) {
  d_query_ids_.assign(query_ids, query_ids + length);
}

uint32_t *AlignerGpuData::GetGpuQuerySeedQueryIds() {
  return thrust::raw_pointer_cast(d_query_ids_.data());
}

void AlignerGpuData::SetGpuConcatenatedQuerySequencePositions(uint32_t *positions,
                                                              size_t length) {
  d_concatenated_query_sequence_positions_.assign(positions, positions + length);
}

uint32_t *AlignerGpuData::GetGpuQuerySeedQueryPositions() {
  return thrust::raw_pointer_cast(d_concatenated_query_sequence_positions_.data());
}

void AlignerGpuData::SetGpuDatabaseSequence(const AlphabetCoder::Code *sequence, size_t length) {
  upload_codes(d_database_sequence_, sequence, length);
}

packed_alphabet_code::PackedAlphabetCode *AlignerGpuData::GetGpuDatabaseSequence() {
  return reinterpret_cast<packed_alphabet_code::PackedAlphabetCode *>(
      reinterpret_cast<uint8_t *>(thrust::raw_pointer_cast(d_database_sequence_.data())) +
      kSequencePad);
}

void AlignerGpuData::SetGpuQueriesSequence(const AlphabetCoder::Code *sequence, size_t length) {
  upload_codes(d_concatenated_query_sequence_, sequence, length);
}

packed_alphabet_code::PackedAlphabetCode *AlignerGpuData::GetGpuQueriesSequence() {
  return reinterpret_cast<packed_alphabet_code::PackedAlphabetCode *>(
      reinterpret_cast<uint8_t *>(
          thrust::raw_pointer_cast(d_concatenated_query_sequence_.data())) +
      kSequencePad);
}

void AlignerGpuData::SetGpuReducedCodeMap(const AlphabetCoder::Code *map, size_t length) {
  d_reduced_code_map_.assign(map, map + length);
}

AlphabetCoder::Code *AlignerGpuData::GetGpuReducedCodeMap() {
  return thrust::raw_pointer_cast(d_reduced_code_map_.data());
}

void AlignerGpuData::SetGpuUngappedExtensionCutoffs(const int *cutoffs, size_t number) {
  d_ungapped_extension_cutoffs_.assign(cutoffs, cutoffs + number);
}

int *AlignerGpuData::GetGpuUngappedExtensionCutoffs() {
  return thrust::raw_pointer_cast(d_ungapped_extension_cutoffs_.data());
}

void AlignerGpuData::SetGpuGappedExtensionTriggers(const int *triggers, size_t number) {
  d_gapped_extension_triggers_.assign(triggers, triggers + number);
}

int *AlignerGpuData::GetGpuGappedExtensionTriggers() {
  return thrust::raw_pointer_cast(d_gapped_extension_triggers_.data());
}

// the (n + 1)^2 device matrix with a zero delimiter row and column
void AlignerGpuData::SetGpuScoreMatrix(const int *score_matrix, size_t number_letters) {
  const size_t n1 = number_letters + 1;
  std::vector<int> m(n1 * n1, 0);
  for (size_t a = 0; a < number_letters; ++a)
    for (size_t b = 0; b < number_letters; ++b)
      m[a * n1 + b] = score_matrix[a * number_letters + b];
  d_score_matrix_.assign(m.begin(), m.end());
}

int *AlignerGpuData::GetGpuScoreMatrix() {
  return thrust::raw_pointer_cast(d_score_matrix_.data());
}

void AlignerGpuData::SetPackedAlphabetCodeSequenceToGpu(
    size_t length, const AlphabetCoder::Code *sequence,
    thrust::device_vector<packed_alphabet_code::PackedAlphabetCode> &d_sequence) {
  upload_codes(d_sequence, sequence, length);
}

// ---- DeviceSeedsMemory (src/device_seeds_memory.h) ------------------------
DeviceSeedsMemory::DeviceSeedsMemory() : size_(0), temp_storage_bytes(0) {}

DeviceSeedsMemory::~DeviceSeedsMemory() {}

int DeviceSeedsMemory::Init(size_t size) {
  size_ = size;
  query_seed_ids_.resize(size);
  query_seed_lengths_.resize(size);
  query_ids_.resize(size);
  query_concatenated_positions_.resize(size);
  database_positions_.resize(size);
  result_values_.resize(size);
  temp_storage_bytes = gzb_ungapped_extender_query_seeds_temp_bytes(size);
  temp_storage_.resize(temp_storage_bytes);
  return 0;
}

size_t DeviceSeedsMemory::GetSize() { return size_; }

// ---- DistanceCalculatorGpu (src/distance_calculator_gpu.h) ----------------
DistanceCalculatorGpu::DistanceCalculatorGpu()
    : subsequence_length_(0),
      d_concatenated_query_sequence_(NULL),
      d_database_sequence_(NULL),
      d_redueced_code_map_(NULL) {
  gzb_distance_calculator *h = nullptr;
  die(gzb_distance_calculator_create(&h), "DistanceCalculatorGpu");
  g_distance.add(this, h);
}

DistanceCalculatorGpu::~DistanceCalculatorGpu() {
  gzb_distance_calculator_destroy(g_distance.take(this));
}

int DistanceCalculatorGpu::SetQueries(
    const packed_alphabet_code::PackedAlphabetCode *query_sequence) {
  d_concatenated_query_sequence_ = query_sequence;
  die(gzb_distance_calculator_set_queries(g_distance.get(this), bytes(query_sequence)),
      "DistanceCalculatorGpu::SetQueries");
  return 0;
}

int DistanceCalculatorGpu::SetDatabase(
    const packed_alphabet_code::PackedAlphabetCode *database_sequence) {
  d_database_sequence_ = database_sequence;
  die(gzb_distance_calculator_set_database(g_distance.get(this), bytes(database_sequence)),
      "DistanceCalculatorGpu::SetDatabase");
  return 0;
}

int DistanceCalculatorGpu::SetReducedCodeMap(const AlphabetCoder::Code *map) {
  d_redueced_code_map_ = map;
  die(gzb_distance_calculator_set_reduced_code_map(g_distance.get(this), map),
      "DistanceCalculatorGpu::SetReducedCodeMap");
  return 0;
}

int DistanceCalculatorGpu::SetSubsequenceLength(uint32_t length) {
  subsequence_length_ = length;
  die(gzb_distance_calculator_set_subsequence_length(g_distance.get(this), length),
      "DistanceCalculatorGpu::SetSubsequenceLength");
  return 0;
}

int DistanceCalculatorGpu::CalculateDistancesAsync(size_t size, uint32_t *query_centers,
                                                   uint32_t *database_centers,
                                                   Distance *distances,
                                                   uint32_t *d_query_centers,
                                                   uint32_t *d_database_centers,
                                                   Distance *d_distances, cudaStream_t &stream) {
  die(gzb_distance_calculator_calculate_distances_async(
          g_distance.get(this), size, query_centers, database_centers, (int8_t *)distances,
          d_query_centers, d_database_centers, (int8_t *)d_distances, (void *)stream),
      "DistanceCalculatorGpu::CalculateDistancesAsync");
  return 0;
}

// ---- UngappedExtenderGpu (src/ungapped_extender_gpu.h) --------------------
UngappedExtenderGpu::UngappedExtenderGpu()
    : number_letters_(0),
      sequence_delimiter_(0),
      d_query_seed_query_ids_(NULL),
      d_query_seed_query_positions_(NULL),
      d_database_sequence_(NULL),
      d_concatenated_query_sequence_(NULL),
      d_score_matrix_(NULL),
      d_ungapped_extension_cutoffs_(NULL),
      d_gapped_extension_triggers_(NULL) {
  gzb_ungapped_extender *h = nullptr;
  die(gzb_ungapped_extender_create(&h), "UngappedExtenderGpu");
  g_ungapped.add(this, h);
}

UngappedExtenderGpu::~UngappedExtenderGpu() {
  gzb_ungapped_extender_destroy(g_ungapped.take(this));
}

int UngappedExtenderGpu::SetQuerySeedDataList(const uint32_t *d_query_ids,
                                              const uint32_t *d_query_positions) {
  d_query_seed_query_ids_ = d_query_ids;
  d_query_seed_query_positions_ = d_query_positions;
  die(gzb_ungapped_extender_set_query_seed_data_list(g_ungapped.get(this), d_query_ids,
                                                     d_query_positions),
      "UngappedExtenderGpu::SetQuerySeedDataList");
  return 0;
}

int UngappedExtenderGpu::SetQueries(
    AlphabetCoder::Code sequence_delimiter,
    const packed_alphabet_code::PackedAlphabetCode *d_concatenated_query_sequence,
    const int *d_ungapped_extension_cutoffs, const int *d_gapped_extension_triggers) {
  sequence_delimiter_ = sequence_delimiter;
  d_concatenated_query_sequence_ = d_concatenated_query_sequence;
  d_ungapped_extension_cutoffs_ = d_ungapped_extension_cutoffs;
  d_gapped_extension_triggers_ = d_gapped_extension_triggers;
  die(gzb_ungapped_extender_set_queries(g_ungapped.get(this), sequence_delimiter,
                                        bytes(d_concatenated_query_sequence),
                                        d_ungapped_extension_cutoffs,
                                        d_gapped_extension_triggers),
      "UngappedExtenderGpu::SetQueries");
  return 0;
}

int UngappedExtenderGpu::SetDatabase(
    const packed_alphabet_code::PackedAlphabetCode *d_database_sequence) {
  d_database_sequence_ = d_database_sequence;
  die(gzb_ungapped_extender_set_database(g_ungapped.get(this), bytes(d_database_sequence)),
      "UngappedExtenderGpu::SetDatabase");
  return 0;
}

int UngappedExtenderGpu::SetScoreMatrix(const int *d_score_matrix, uint32_t number_letters) {
  number_letters_ = number_letters;
  d_score_matrix_ = d_score_matrix;
  die(gzb_ungapped_extender_set_score_matrix(g_ungapped.get(this), d_score_matrix,
                                             number_letters),
      "UngappedExtenderGpu::SetScoreMatrix");
  return 0;
}

int UngappedExtenderGpu::SetQuerySeeds(size_t query_seeds_size, size_t size,
                                       uint32_t *query_seed_ids, uint32_t *query_seed_starts,
                                       size_t temp_storage_bytes, void *d_temp_storage,
                                       uint32_t *d_query_seed_ids,
                                       uint32_t *d_query_seed_starts, uint32_t *d_query_ids,
                                       uint32_t *d_query_concatenated_positions,
                                       uint32_t *temp_array, cudaStream_t &stream) const {
  die(gzb_ungapped_extender_set_query_seeds(
          g_ungapped.get(this), query_seeds_size, size, query_seed_ids, query_seed_starts,
          temp_storage_bytes, d_temp_storage, d_query_seed_ids, d_query_seed_starts,
          d_query_ids, d_query_concatenated_positions, temp_array, (void *)stream),
      "UngappedExtenderGpu::SetQuerySeeds");
  return 0;
}

int UngappedExtenderGpu::ExtendWithTriggerAsync(
    size_t size, uint32_t *query_ids, uint32_t *query_concatenated_positions,
    uint32_t *database_positions, char *flags, uint32_t *d_query_ids,
    uint32_t *d_query_concatenated_positions, uint32_t *d_database_positions, char *d_flags,
    int *d_temp_array, cudaStream_t &stream) const {
  die(gzb_ungapped_extender_extend_with_trigger_async(
          g_ungapped.get(this), size, query_ids, query_concatenated_positions,
          database_positions, (int8_t *)flags, d_query_ids, d_query_concatenated_positions,
          d_database_positions, (int8_t *)d_flags, d_temp_array, (void *)stream),
      "UngappedExtenderGpu::ExtendWithTriggerAsync");
  return 0;
}

// The score-returning overload and ExtendOneSideAsync have no caller in the
// reference's aligner (src/ungapped_extender_gpu.h:47-64).
int UngappedExtenderGpu::ExtendWithTriggerAsync(size_t, uint32_t *, uint32_t *, size_t,
                                                uint32_t *, uint32_t *, uint32_t *, int *,
                                                uint32_t *, uint32_t *, size_t, void *,
                                                uint32_t *, uint32_t *, uint32_t *, int *,
                                                cudaStream_t &) const {
  fprintf(stderr, "UngappedExtenderGpu: the score-returning ExtendWithTriggerAsync is not "
                  "provided by libghostz_b200\n");
  exit(1);
}

int UngappedExtenderGpu::ExtendOneSideAsync(size_t, bool, uint32_t *, uint32_t *, uint32_t *,
                                            int *, uint32_t *, uint32_t *, uint32_t *, int *,
                                            cudaStream_t &) const {
  fprintf(stderr, "UngappedExtenderGpu: ExtendOneSideAsync is not provided by "
                  "libghostz_b200\n");
  exit(1);
}

// ---- GappedExtenderGpu (src/gapped_extender_gpu.h) ------------------------
GappedExtenderGpu::GappedExtenderGpu()
    : number_letters_(0),
      gap_open_(0),
      gap_extention_(0),
      cutoff_(0),
      sequence_delimiter_(0),
      d_database_sequence_(NULL),
      d_concatenated_query_sequence_(NULL),
      d_score_matrix_(NULL),
      d_ungapped_extension_cutoffs_(NULL) {
  gzb_gapped_extender *h = nullptr;
  die(gzb_gapped_extender_create(&h), "GappedExtenderGpu");
  g_gapped.add(this, h);
}

GappedExtenderGpu::~GappedExtenderGpu() { gzb_gapped_extender_destroy(g_gapped.take(this)); }

int GappedExtenderGpu::SetQueries(
    AlphabetCoder::Code sequence_delimiter,
    const packed_alphabet_code::PackedAlphabetCode *d_concatenated_query_sequence) {
  sequence_delimiter_ = sequence_delimiter;
  d_concatenated_query_sequence_ = d_concatenated_query_sequence;
  die(gzb_gapped_extender_set_queries(g_gapped.get(this), sequence_delimiter,
                                      bytes(d_concatenated_query_sequence)),
      "GappedExtenderGpu::SetQueries");
  return 0;
}

int GappedExtenderGpu::SetDatabase(
    const packed_alphabet_code::PackedAlphabetCode *d_database_sequence) {
  d_database_sequence_ = d_database_sequence;
  die(gzb_gapped_extender_set_database(g_gapped.get(this), bytes(d_database_sequence)),
      "GappedExtenderGpu::SetDatabase");
  return 0;
}

int GappedExtenderGpu::SetScoreParameters(const int *d_score_matrix, uint32_t number_letters,
                                          int gap_open, int gap_extention, int cutoff) {
  number_letters_ = number_letters;
  d_score_matrix_ = d_score_matrix;
  gap_open_ = gap_open;
  gap_extention_ = gap_extention;
  cutoff_ = cutoff;
  die(gzb_gapped_extender_set_score_parameters(g_gapped.get(this), d_score_matrix,
                                               number_letters, gap_open, gap_extention, cutoff),
      "GappedExtenderGpu::SetScoreParameters");
  return 0;
}

int GappedExtenderGpu::ConvertToGappedExtensionSeedsAsync(
    size_t size, bool reverse, uint32_t *seed_positions,
    uint32_t *query_concatenated_positions, uint32_t *database_positions,
    uint32_t *d_seed_positions, uint32_t *d_temp_array,
    uint32_t *d_query_concatenated_positions, uint32_t *d_database_positions,
    cudaStream_t &stream) const {
  die(gzb_gapped_extender_convert_to_gapped_extension_seeds_async(
          g_gapped.get(this), size, reverse ? 1 : 0, seed_positions,
          query_concatenated_positions, database_positions, d_seed_positions, d_temp_array,
          d_query_concatenated_positions, d_database_positions, (void *)stream),
      "GappedExtenderGpu::ConvertToGappedExtensionSeedsAsync");
  return 0;
}

int GappedExtenderGpu::ExtendOneSideScoreOnlyAsync(
    size_t size, bool reverse, uint32_t *query_concatenated_positions,
    uint32_t *database_positions, int *scores, uint32_t *d_query_concatenated_positions,
    uint32_t *d_database_positions, int *d_scores, cudaStream_t &stream) const {
  die(gzb_gapped_extender_extend_one_side_score_only_async(
          g_gapped.get(this), size, reverse ? 1 : 0, query_concatenated_positions,
          database_positions, scores, d_query_concatenated_positions, d_database_positions,
          d_scores, (void *)stream),
      "GappedExtenderGpu::ExtendOneSideScoreOnlyAsync");
  return 0;
}
