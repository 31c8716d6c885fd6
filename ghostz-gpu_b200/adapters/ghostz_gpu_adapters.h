// ghostz_gpu_adapters.h -- the reference's GPU operator classes, header only,
// implemented over the C ABI of libghostz_b200.so.
//
// The classes keep the names, method names and argument order of
// DistanceCalculatorGpu (src/distance_calculator_gpu.h:18-40),
// UngappedExtenderGpu (src/ungapped_extender_gpu.h:21-76) and
// GappedExtenderGpu (src/gapped_extender_gpu.h:19-60), so the reference's
// GpuStreamRunner / AlignerGpuPresearchThread call sites compile unchanged
// against them.  Two differences a maintainer adjusts in AlignerGpuData:
//   * device sequences are one byte per residue code (AlphabetCoder::Code)
//     with at least 64 readable bytes before and after them, instead of the
//     5-bit PackedAlphabetCode words;
//   * errors come back as non-zero return codes (the message is in
//     gzb_last_error()) instead of exit(1); the adapters forward them.
// Scores and positions are bit-identical to the CPU GappedExtender /
// UngappedExtender / DistanceCalculator, without the reference GPU kernel's
// 128-residue query limit.
#ifndef GHOSTZ_GPU_ADAPTERS_H_
#define GHOSTZ_GPU_ADAPTERS_H_

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <istream>
#include <iterator>
#include <vector>

#include "ghostz_b200.h"

namespace ghostz_b200 {

typedef uint8_t Code;        // AlphabetCoder::Code
typedef char Distance;       // DistanceCalculator::Distance

class DistanceCalculatorGpu {
 public:
  DistanceCalculatorGpu() : h_(0) { gzb_distance_calculator_create(&h_); }
  virtual ~DistanceCalculatorGpu() { gzb_distance_calculator_destroy(h_); }
  int SetQueries(const Code *d_query_sequence) {
    return gzb_distance_calculator_set_queries(h_, d_query_sequence);
  }
  int SetDatabase(const Code *d_database_sequence) {
    return gzb_distance_calculator_set_database(h_, d_database_sequence);
  }
  int SetReducedCodeMap(const Code *d_reduced_code_map) {
    return gzb_distance_calculator_set_reduced_code_map(h_, d_reduced_code_map);
  }
  int SetSubsequenceLength(uint32_t length) {
    return gzb_distance_calculator_set_subsequence_length(h_, length);
  }
  int CalculateDistancesAsync(size_t size, uint32_t *query_concatenated_centers,
                              uint32_t *database_centers, Distance *distances,
                              uint32_t *d_query_concatenated_centers,
                              uint32_t *d_database_centers, Distance *d_distances,
                              cudaStream_t &stream) {
    return gzb_distance_calculator_calculate_distances_async(
        h_, size, query_concatenated_centers, database_centers, (int8_t *)distances,
        d_query_concatenated_centers, d_database_centers, (int8_t *)d_distances,
        (void *)stream);
  }

 private:
  DistanceCalculatorGpu(const DistanceCalculatorGpu &);
  DistanceCalculatorGpu &operator=(const DistanceCalculatorGpu &);
  gzb_distance_calculator *h_;
};

class UngappedExtenderGpu {
 public:
  UngappedExtenderGpu() : h_(0) { gzb_ungapped_extender_create(&h_); }
  virtual ~UngappedExtenderGpu() { gzb_ungapped_extender_destroy(h_); }
  int SetQuerySeedDataList(const uint32_t *d_query_ids, const uint32_t *d_query_positions) {
    return gzb_ungapped_extender_set_query_seed_data_list(h_, d_query_ids, d_query_positions);
  }
  int SetQueries(Code sequence_delimiter, const Code *d_concatenated_query_sequence,
                 const int *d_ungapped_extension_cutoffs,
                 const int *d_gapped_extension_triggers) {
    return gzb_ungapped_extender_set_queries(h_, sequence_delimiter,
                                             d_concatenated_query_sequence,
                                             d_ungapped_extension_cutoffs,
                                             d_gapped_extension_triggers);
  }
  int SetDatabase(const Code *d_database_sequence) {
    return gzb_ungapped_extender_set_database(h_, d_database_sequence);
  }
  // d_score_matrix: (number_letters + 1)^2 with a zero delimiter row/column
  int SetScoreMatrix(const int *d_score_matrix, uint32_t number_letters) {
    return gzb_ungapped_extender_set_score_matrix(h_, d_score_matrix, number_letters);
  }
  int SetQuerySeeds(size_t query_seeds_size, size_t size, uint32_t *query_seed_ids,
                    uint32_t *query_seed_starts, size_t temp_storage_bytes,
                    void *d_temp_storage, uint32_t *d_query_seed_ids,
                    uint32_t *d_query_seed_starts, uint32_t *d_query_ids,
                    uint32_t *d_query_concatenated_positions, uint32_t *temp_array,
                    cudaStream_t &stream) const {
    return gzb_ungapped_extender_set_query_seeds(
        h_, query_seeds_size, size, query_seed_ids, query_seed_starts, temp_storage_bytes,
        d_temp_storage, d_query_seed_ids, d_query_seed_starts, d_query_ids,
        d_query_concatenated_positions, temp_array, (void *)stream);
  }
  int ExtendWithTriggerAsync(size_t size, uint32_t *query_ids,
                             uint32_t *query_concatenated_positions,
                             uint32_t *database_positions, char *flags, uint32_t *d_query_ids,
                             uint32_t *d_query_concatenated_positions,
                             uint32_t *d_database_positions, char *d_flags, int *d_temp_array,
                             cudaStream_t &stream) const {
    return gzb_ungapped_extender_extend_with_trigger_async(
        h_, size, query_ids, query_concatenated_positions, database_positions,
        (int8_t *)flags, d_query_ids, d_query_concatenated_positions, d_database_positions,
        (int8_t *)d_flags, d_temp_array, (void *)stream);
  }
  // temp bytes SetQuerySeeds needs (the reference sizes a CUB scan for this)
  static size_t QuerySeedsTempStorageBytes(size_t size) {
    return gzb_ungapped_extender_query_seeds_temp_bytes(size);
  }

 private:
  UngappedExtenderGpu(const UngappedExtenderGpu &);
  UngappedExtenderGpu &operator=(const UngappedExtenderGpu &);
  gzb_ungapped_extender *h_;
};

class GappedExtenderGpu {
 public:
  static const int kInitScore = -(1 << 10);
  GappedExtenderGpu() : h_(0) { gzb_gapped_extender_create(&h_); }
  virtual ~GappedExtenderGpu() { gzb_gapped_extender_destroy(h_); }
  int SetQueries(Code sequence_delimiter, const Code *d_concatenated_query_sequence) {
    return gzb_gapped_extender_set_queries(h_, sequence_delimiter,
                                           d_concatenated_query_sequence);
  }
  int SetDatabase(const Code *d_database_sequence) {
    return gzb_gapped_extender_set_database(h_, d_database_sequence);
  }
  int SetScoreParameters(const int *d_score_matrix, uint32_t number_letters, int gap_open,
                         int gap_extention, int cutoff) {
    return gzb_gapped_extender_set_score_parameters(h_, d_score_matrix, number_letters,
                                                    gap_open, gap_extention, cutoff);
  }
  int ConvertToGappedExtensionSeedsAsync(size_t size, bool reverse, uint32_t *seed_positions,
                                         uint32_t *query_concatenated_positions,
                                         uint32_t *database_positions,
                                         uint32_t *d_seed_positions, uint32_t *d_temp_array,
                                         uint32_t *d_query_concatenated_positions,
                                         uint32_t *d_database_positions,
                                         cudaStream_t &stream) const {
    return gzb_gapped_extender_convert_to_gapped_extension_seeds_async(
        h_, size, reverse ? 1 : 0, seed_positions, query_concatenated_positions,
        database_positions, d_seed_positions, d_temp_array, d_query_concatenated_positions,
        d_database_positions, (void *)stream);
  }
  int ExtendOneSideScoreOnlyAsync(size_t size, bool reverse,
                                  uint32_t *query_concatenated_positions,
                                  uint32_t *database_positions, int *scores,
                                  uint32_t *d_query_concatenated_positions,
                                  uint32_t *d_database_positions, int *d_scores,
                                  cudaStream_t &stream) const {
    return gzb_gapped_extender_extend_one_side_score_only_async(
        h_, size, reverse ? 1 : 0, query_concatenated_positions, database_positions, scores,
        d_query_concatenated_positions, d_database_positions, d_scores, (void *)stream);
  }

 private:
  GappedExtenderGpu(const GappedExtenderGpu &);
  GappedExtenderGpu &operator=(const GappedExtenderGpu &);
  gzb_gapped_extender *h_;
};

// The counterpart of SeedSearcherDatabaseParameters::Build(sequence,
// length, istream) (src/seed_searcher_database_parameters.cpp:321-337): a
// chunk and the index the reference's `db` command saved for it (the
// chunk's `.sdp` stream) made resident in `engine`, the index converted on
// the host instead of being rebuilt.  offsets: first residue of each of the
// number_sequences sequences, then the chunk length.  Unlike the reference,
// which reads only its own record, this reads `in` to its end and refuses
// trailing bytes: the stream must hold exactly one chunk's `.sdp` (open the
// chunk's own file, or hand over a stream limited to its record).
inline int LoadChunkWithReferenceIndex(gzb_engine *engine, const gzb_params &params,
                                       int32_t chunk_id, const Code *sequence,
                                       uint64_t length, const uint32_t *offsets,
                                       uint32_t number_sequences, std::istream &sdp,
                                       cudaStream_t stream) {
  std::vector<char> bytes((std::istreambuf_iterator<char>(sdp)),
                          std::istreambuf_iterator<char>());
  uint64_t n = 0;
  int rc = gzb_index_blob_from_reference(&params, bytes.data(), bytes.size(), sequence, length,
                                         offsets, number_sequences, 0, 0, &n);
  if (rc) return rc;
  std::vector<uint8_t> blob(n);
  rc = gzb_index_blob_from_reference(&params, bytes.data(), bytes.size(), sequence, length,
                                     offsets, number_sequences, blob.data(), n, &n);
  if (rc) return rc;
  return gzb_engine_set_database_with_index(engine, chunk_id, sequence, length, offsets,
                                            number_sequences, blob.data(), n, (void *)stream);
}

}  // namespace ghostz_b200

#endif  // GHOSTZ_GPU_ADAPTERS_H_
