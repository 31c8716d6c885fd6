/*
 * CPU stand-ins for the device layer of the reference's GPU aligner (test
 * infrastructure only).
 *
 * The reference's GPU search (`ghostz-gpu aln -g N`, src/aligner_gpu.cpp,
 * src/aligner_gpu_presearch_thread.cpp, src/seed_searcher_gpu*.cpp,
 * src/gpu_stream_*.cpp) is host C++ that composes the seed search, seed
 * lists, chain filter, extension seed lists, result merge and build results
 * around three device operators and a device data holder.  The oracle's
 * reference build compiles that host code unchanged and links it with the
 * definitions in this file, which keep the reference's class declarations
 * (src/distance_calculator_gpu.h, src/ungapped_extender_gpu.h,
 * src/gapped_extender_gpu.h, src/aligner_gpu_data.h,
 * src/device_seeds_memory.h) and compute each operator's result on the CPU
 * with the reference's own CPU arithmetic:
 *
 *  - DistanceCalculatorGpu: DistanceCalculator::CalculateDistance
 *    (src/distance_calculator.cpp:35-54) over the unpacked sequences;
 *  - UngappedExtenderGpu::ExtendWithTriggerAsync: the flag of
 *    SeedSearcher::UngappedExtend (src/seed_searcher.h:133-158), i.e. the
 *    reverse UngappedExtender::ExtendOneSideScoreOnly, then the forward one
 *    while the sum is at most the trigger, flag = sum > trigger (the decision
 *    UngappedExtendKernel makes, src/ungapped_extender_gpu.cu:192-330);
 *  - UngappedExtenderGpu::SetQuerySeeds: the run-length expansion of
 *    src/ungapped_extender_gpu.cu:818-852 (starts scattered, max-scan,
 *    gather of the query-seed data);
 *  - GappedExtenderGpu: ConvertToGappedExtensionSeeds (a gather,
 *    src/gapped_extender_gpu.cu:719-733 and :768-801) and
 *    GappedExtender::ExtendOneSide without edit blocks
 *    (src/gapped_extender.cpp:306-471) for ExtendOneSideScoreOnlyAsync,
 *    positions moved to the best end as ExtendOneSideScoreOnlyKernel does
 *    (src/gapped_extender_gpu.cu:545-717).  The reference kernel caches at
 *    most 128 query codes (kMaxSequence0Length); the stand-in extends over
 *    the whole remainder, as the reference's CPU extender does;
 *  - AlignerGpuData: the same packed layout (12 five-bit codes per 64-bit
 *    word behind 4 words of padding, src/aligner_gpu_data.cu:129-147), with
 *    the unpacked codes kept beside each packed array so the operators read
 *    them directly.
 *
 * Every "device" pointer is host memory (Thrust's device system is the
 * host's in this build) and every operation finishes before its call
 * returns, so stream synchronisation is a no-op (cuda_host.cpp).
 */
#include <stdint.h>

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "aligner_gpu_data.h"
#include "device_seeds_memory.h"
#include "distance_calculator.h"
#include "distance_calculator_gpu.h"
#include "gapped_extender.h"
#include "gapped_extender_gpu.h"
#include "score_matrix.h"
#include "ungapped_extender.h"
#include "ungapped_extender_gpu.h"

namespace {

typedef AlphabetCoder::Code Code;

/* unpacked codes of every packed sequence handed out, by packed pointer */
std::mutex g_registry_mutex;
std::map<const void *, std::vector<Code> > g_registry;

void RegisterCodes(const void *packed, const Code *codes, size_t length) {
  std::lock_guard<std::mutex> lock(g_registry_mutex);
  g_registry[packed].assign(codes, codes + length);
}

const Code *CodesOf(const void *packed) {
  std::lock_guard<std::mutex> lock(g_registry_mutex);
  std::map<const void *, std::vector<Code> >::const_iterator it =
      g_registry.find(packed);
  if (it == g_registry.end()) {
    fprintf(stderr, "host operators: unknown packed sequence %p\n", packed);
    abort();
  }
  return it->second.empty() ? NULL : &it->second[0];
}

/* the n x n matrix of the device's (n + 1)^2 layout (delimiter row and
 * column zero, src/aligner_gpu_data.cu:110-124) as a ScoreMatrix */
ScoreMatrix MatrixOf(const int *device_matrix, uint32_t number_letters) {
  std::vector<int> m(number_letters * number_letters);
  for (uint32_t a = 0; a < number_letters; ++a)
    for (uint32_t b = 0; b < number_letters; ++b)
      m[a * number_letters + b] = device_matrix[a * (number_letters + 1) + b];
  return ScoreMatrix("device", &m[0], number_letters);
}

void Copy(void *dst, const void *src, size_t bytes) {
  if (dst != src && bytes) memmove(dst, src, bytes);
}

}  // namespace

/* ---- AlignerGpuData (src/aligner_gpu_data.h) --------------------------- */
AlignerGpuData::AlignerGpuData() : gpu_id_(0) {}
AlignerGpuData::AlignerGpuData(int gpu_id) : gpu_id_(gpu_id) {}
AlignerGpuData::~AlignerGpuData() {}
void AlignerGpuData::SetGpuId(int gpu_id) { gpu_id_ = gpu_id; }
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
void AlignerGpuData::SetGpuDatabaseSequence(const AlphabetCoder::Code *sequence,
                                            size_t length) {
  SetPackedAlphabetCodeSequenceToGpu(length, sequence, d_database_sequence_);
  RegisterCodes(thrust::raw_pointer_cast(d_database_sequence_.data()), sequence, length);
}
packed_alphabet_code::PackedAlphabetCode *AlignerGpuData::GetGpuDatabaseSequence() {
  return thrust::raw_pointer_cast(d_database_sequence_.data());
}
void AlignerGpuData::SetGpuQueriesSequence(const AlphabetCoder::Code *sequence,
                                           size_t length) {
  SetPackedAlphabetCodeSequenceToGpu(length, sequence, d_concatenated_query_sequence_);
  RegisterCodes(thrust::raw_pointer_cast(d_concatenated_query_sequence_.data()), sequence,
                length);
}
packed_alphabet_code::PackedAlphabetCode *AlignerGpuData::GetGpuQueriesSequence() {
  return thrust::raw_pointer_cast(d_concatenated_query_sequence_.data());
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
void AlignerGpuData::SetGpuScoreMatrix(const int *score_matrix, size_t number_letters) {
  const size_t n1 = number_letters + 1;
  d_score_matrix_.assign(n1 * n1, 0);
  for (size_t a = 0; a < number_letters; ++a)
    for (size_t b = 0; b < number_letters; ++b)
      d_score_matrix_[a * n1 + b] = score_matrix[a * number_letters + b];
}
int *AlignerGpuData::GetGpuScoreMatrix() {
  return thrust::raw_pointer_cast(d_score_matrix_.data());
}
void AlignerGpuData::SetPackedAlphabetCodeSequenceToGpu(
    size_t length, const AlphabetCoder::Code *sequence,
    thrust::device_vector<packed_alphabet_code::PackedAlphabetCode> &d_packed) {
  const size_t n = packed_alphabet_code::GetPackedAlphabetCodeSequenceLength(length);
  temp_packed_alphabet_code_sequence_.assign(n, 0);
  packed_alphabet_code::PackAlphabetCodeSequence(sequence, length,
                                                 &temp_packed_alphabet_code_sequence_[0]);
  const size_t pad = cuda_common::kMaxLoadLength;
  if (d_packed.size() < n + 2 * pad) d_packed.resize(n + 2 * pad);
  for (size_t i = 0; i < n; ++i) d_packed[pad + i] = temp_packed_alphabet_code_sequence_[i];
}

/* ---- DeviceSeedsMemory (src/device_seeds_memory.h) --------------------- */
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
  temp_storage_bytes = 16;  // the stand-in scan needs no scratch
  temp_storage_.resize(temp_storage_bytes);
  return 0;
}
size_t DeviceSeedsMemory::GetSize() { return size_; }

/* ---- DistanceCalculatorGpu (src/distance_calculator_gpu.h) ------------- */
DistanceCalculatorGpu::DistanceCalculatorGpu()
    : subsequence_length_(0),
      d_concatenated_query_sequence_(NULL),
      d_database_sequence_(NULL),
      d_redueced_code_map_(NULL) {}
DistanceCalculatorGpu::~DistanceCalculatorGpu() {}
int DistanceCalculatorGpu::SetQueries(
    const packed_alphabet_code::PackedAlphabetCode *query_sequence) {
  d_concatenated_query_sequence_ = query_sequence;
  return 0;
}
int DistanceCalculatorGpu::SetDatabase(
    const packed_alphabet_code::PackedAlphabetCode *database_sequence) {
  d_database_sequence_ = database_sequence;
  return 0;
}
int DistanceCalculatorGpu::SetReducedCodeMap(const AlphabetCoder::Code *map) {
  d_redueced_code_map_ = map;
  return 0;
}
int DistanceCalculatorGpu::SetSubsequenceLength(uint32_t length) {
  subsequence_length_ = length;
  return 0;
}
int DistanceCalculatorGpu::CalculateDistancesAsync(
    size_t size, uint32_t *query_concatenated_centers, uint32_t *database_centers,
    Distance *distances, uint32_t *d_query_concatenated_centers,
    uint32_t *d_database_centers, Distance *d_distances, cudaStream_t &stream) {
  (void)stream;
  Copy(d_query_concatenated_centers, query_concatenated_centers, sizeof(uint32_t) * size);
  Copy(d_database_centers, database_centers, sizeof(uint32_t) * size);
  DistanceCalculator calc;
  calc.SetQueries(CodesOf(d_concatenated_query_sequence_));
  calc.SetDatabase(CodesOf(d_database_sequence_));
  calc.SetReducedCodeMap(d_redueced_code_map_);
  for (size_t i = 0; i < size; ++i)
    d_distances[i] = calc.CalculateDistance(d_query_concatenated_centers[i],
                                            d_database_centers[i], subsequence_length_);
  Copy(distances, d_distances, sizeof(Distance) * size);
  return 0;
}

/* ---- UngappedExtenderGpu (src/ungapped_extender_gpu.h) ----------------- */
UngappedExtenderGpu::UngappedExtenderGpu()
    : number_letters_(0),
      sequence_delimiter_(0),
      d_query_seed_query_ids_(NULL),
      d_query_seed_query_positions_(NULL),
      d_database_sequence_(NULL),
      d_concatenated_query_sequence_(NULL),
      d_score_matrix_(NULL),
      d_ungapped_extension_cutoffs_(NULL),
      d_gapped_extension_triggers_(NULL) {}
UngappedExtenderGpu::~UngappedExtenderGpu() {}
int UngappedExtenderGpu::SetQuerySeedDataList(const uint32_t *d_query_ids,
                                              const uint32_t *d_query_positions) {
  d_query_seed_query_ids_ = d_query_ids;
  d_query_seed_query_positions_ = d_query_positions;
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
  return 0;
}
int UngappedExtenderGpu::SetDatabase(
    const packed_alphabet_code::PackedAlphabetCode *d_database_sequence) {
  d_database_sequence_ = d_database_sequence;
  return 0;
}
int UngappedExtenderGpu::SetScoreMatrix(const int *d_score_matrix, uint32_t number_letters) {
  number_letters_ = number_letters;
  d_score_matrix_ = d_score_matrix;
  return 0;
}

int UngappedExtenderGpu::SetQuerySeeds(size_t query_seeds_size, size_t size,
                                       uint32_t *query_seed_ids, uint32_t *query_seed_starts,
                                       size_t temp_storage_bytes, void *d_temp_storage,
                                       uint32_t *d_query_seed_ids,
                                       uint32_t *d_query_seed_starts, uint32_t *d_query_ids,
                                       uint32_t *d_query_concatenated_positions,
                                       uint32_t *temp_array, cudaStream_t &stream) const {
  (void)temp_storage_bytes;
  (void)d_temp_storage;
  (void)stream;
  Copy(d_query_seed_starts, query_seed_starts, sizeof(uint32_t) * query_seeds_size);
  /* every seed's index into the run list: run i covers the seeds from its
   * start up to the next run's start (zero-filled, starts scattered, then an
   * inclusive max-scan) */
  std::vector<uint32_t> run_of(size, 0);
  for (size_t i = 0; i < query_seeds_size; ++i)
    if (d_query_seed_starts[i] < size) run_of[d_query_seed_starts[i]] = (uint32_t)i;
  for (size_t s = 1; s < size; ++s)
    if (run_of[s] < run_of[s - 1]) run_of[s] = run_of[s - 1];
  if (size) Copy(temp_array, &run_of[0], sizeof(uint32_t) * size);
  Copy(d_query_seed_ids, query_seed_ids, sizeof(uint32_t) * query_seeds_size);
  for (size_t s = 0; s < size; ++s) {
    const uint32_t id = d_query_seed_ids[run_of[s]];
    d_query_ids[s] = d_query_seed_query_ids_[id];
    d_query_concatenated_positions[s] = d_query_seed_query_positions_[id];
  }
  return 0;
}

int UngappedExtenderGpu::ExtendWithTriggerAsync(
    size_t size, uint32_t *query_ids, uint32_t *query_concatenated_positions,
    uint32_t *database_positions, char *flags, uint32_t *d_query_ids,
    uint32_t *d_query_concatenated_positions, uint32_t *d_database_positions, char *d_flags,
    int *d_temp_array, cudaStream_t &stream) const {
  (void)d_temp_array;
  (void)stream;
  if (query_ids) Copy(d_query_ids, query_ids, sizeof(uint32_t) * size);
  if (query_concatenated_positions)
    Copy(d_query_concatenated_positions, query_concatenated_positions,
         sizeof(uint32_t) * size);
  Copy(d_database_positions, database_positions, sizeof(uint32_t) * size);
  const Code *query = CodesOf(d_concatenated_query_sequence_);
  const Code *db = CodesOf(d_database_sequence_);
  const ScoreMatrix m = MatrixOf(d_score_matrix_, number_letters_);
  for (size_t i = 0; i < size; ++i) {
    const uint32_t qid = d_query_ids[i];
    const uint32_t qp = d_query_concatenated_positions[i];
    const uint32_t dp = d_database_positions[i];
    const int cutoff = d_ungapped_extension_cutoffs_[qid];
    const int trigger = d_gapped_extension_triggers_[qid];
    int sum = 0, score = 0;
    UngappedExtender::ExtendOneSideScoreOnly(query + qp - 1, db + dp - 1, sequence_delimiter_,
                                             true, m, cutoff, &score);
    sum += score;
    if (sum <= trigger) {
      UngappedExtender::ExtendOneSideScoreOnly(query + qp, db + dp, sequence_delimiter_, false,
                                               m, cutoff, &score);
      sum += score;
    }
    d_flags[i] = sum > trigger ? 1 : 0;
  }
  Copy(flags, d_flags, sizeof(char) * size);
  return 0;
}

int UngappedExtenderGpu::ExtendWithTriggerAsync(
    size_t, uint32_t *, uint32_t *, size_t, uint32_t *, uint32_t *, uint32_t *, int *,
    uint32_t *, uint32_t *, size_t, void *, uint32_t *, uint32_t *, uint32_t *, int *,
    cudaStream_t &) const {
  fprintf(stderr, "host operators: the score-returning ExtendWithTriggerAsync is unused\n");
  abort();
}

int UngappedExtenderGpu::ExtendOneSideAsync(size_t, bool, uint32_t *, uint32_t *, uint32_t *,
                                            int *, uint32_t *, uint32_t *, uint32_t *, int *,
                                            cudaStream_t &) const {
  fprintf(stderr, "host operators: ExtendOneSideAsync is unused\n");
  abort();
}

/* ---- GappedExtenderGpu (src/gapped_extender_gpu.h) --------------------- */
GappedExtenderGpu::GappedExtenderGpu()
    : number_letters_(0),
      gap_open_(0),
      gap_extention_(0),
      cutoff_(0),
      sequence_delimiter_(0),
      d_database_sequence_(NULL),
      d_concatenated_query_sequence_(NULL),
      d_score_matrix_(NULL),
      d_ungapped_extension_cutoffs_(NULL) {}
GappedExtenderGpu::~GappedExtenderGpu() {}
int GappedExtenderGpu::SetQueries(
    AlphabetCoder::Code sequence_delimiter,
    const packed_alphabet_code::PackedAlphabetCode *d_concatenated_query_sequence) {
  sequence_delimiter_ = sequence_delimiter;
  d_concatenated_query_sequence_ = d_concatenated_query_sequence;
  return 0;
}
int GappedExtenderGpu::SetDatabase(
    const packed_alphabet_code::PackedAlphabetCode *d_database_sequence) {
  d_database_sequence_ = d_database_sequence;
  return 0;
}
int GappedExtenderGpu::SetScoreParameters(const int *d_score_matrix, uint32_t number_letters,
                                          int gap_open, int gap_extention, int cutoff) {
  number_letters_ = number_letters;
  d_score_matrix_ = d_score_matrix;
  gap_open_ = gap_open;
  gap_extention_ = gap_extention;
  cutoff_ = cutoff;
  return 0;
}

int GappedExtenderGpu::ConvertToGappedExtensionSeedsAsync(
    size_t size, bool reverse, uint32_t *seed_positions,
    uint32_t *query_concatenated_positions, uint32_t *database_positions,
    uint32_t *d_seed_positions, uint32_t *d_temp_array,
    uint32_t *d_query_concatenated_positions, uint32_t *d_database_positions,
    cudaStream_t &stream) const {
  (void)reverse;
  (void)stream;
  /* the first `size` host positions are staged in d_temp_array and
   * gathered at the seed positions, once for the query and once for the
   * database */
  Copy(d_seed_positions, seed_positions, sizeof(uint32_t) * size);
  Copy(d_temp_array, query_concatenated_positions, sizeof(uint32_t) * size);
  for (size_t i = 0; i < size; ++i)
    d_query_concatenated_positions[i] = d_temp_array[d_seed_positions[i]];
  Copy(d_temp_array, database_positions, sizeof(uint32_t) * size);
  for (size_t i = 0; i < size; ++i) d_database_positions[i] = d_temp_array[d_seed_positions[i]];
  return 0;
}

int GappedExtenderGpu::ExtendOneSideScoreOnlyAsync(
    size_t size, bool reverse, uint32_t *query_concatenated_positions,
    uint32_t *database_positions, int *scores, uint32_t *d_query_concatenated_positions,
    uint32_t *d_database_positions, int *d_scores, cudaStream_t &stream) const {
  (void)stream;
  const Code *query = CodesOf(d_concatenated_query_sequence_);
  const Code *db = CodesOf(d_database_sequence_);
  const ScoreMatrix m = MatrixOf(d_score_matrix_, number_letters_);
  GappedExtender extender;
  for (size_t i = 0; i < size; ++i) {
    const uint32_t qp = d_query_concatenated_positions[i];
    const uint32_t dp = d_database_positions[i];
    /* the query codes up to its delimiter in the extension's direction, as
     * the reference's CPU presearch passes them
     * (src/aligner_presearch_thread.cpp:336-355) */
    uint32_t length = 0;
    if (reverse) {
      while (query[qp - length] != sequence_delimiter_) ++length;
    } else {
      while (query[qp + length] != sequence_delimiter_) ++length;
      ++length;
    }
    int best = 0, best_q = 0, best_d = 0;
    extender.ExtendOneSide(query + qp, length, db + dp, sequence_delimiter_, reverse, m,
                           gap_open_, gap_extention_, cutoff_, &best, &best_q, &best_d, NULL);
    d_query_concatenated_positions[i] = qp + (uint32_t)best_q;
    d_database_positions[i] = dp + (uint32_t)best_d;
    d_scores[i] = best;
  }
  Copy(query_concatenated_positions, d_query_concatenated_positions, sizeof(uint32_t) * size);
  Copy(database_positions, d_database_positions, sizeof(uint32_t) * size);
  Copy(scores, d_scores, sizeof(int) * size);
  return 0;
}
