// gzb_blob.h -- the device index cache's blob format, shared by the engine
// (export / import of a chunk's device index) and the converter of the
// reference's on-disk seed-searcher index.  Host code only.
#pragma once

#include <cstddef>
#include <cstdint>

#include "ghostz_b200.h"

namespace gzb {

// Blob: IndexHeader, then the ten index arrays in index_array_sizes order,
// each padded to 8 bytes.
constexpr uint64_t kIndexMagic = 0x3130584449425a47ull;  // "GZBIDX01"

struct IndexHeader {
  uint64_t magic;
  uint64_t fingerprint;  // parameters the index depends on
  uint64_t db_len, nseq, db_check;
  uint64_t n_nc_keys, n_nc_values, n_rep_keys, n_reps, n_members;
};

inline uint64_t fnv1a(uint64_t h, const void *p, size_t n) {
  const uint8_t *b = (const uint8_t *)p;
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  return h;
}

// the parameters the index build reads (hash, similarity windows, clustering)
inline uint64_t params_fingerprint(const gzb_params &p) {
  uint64_t h = 0xcbf29ce484222325ull;
  const int32_t v[] = {p.delimiter, p.number_letters, p.map_size, p.max_indexing_code,
                       p.seed_threshold, p.max_hash_length, p.min_hash_length,
                       p.subsequence_length, p.max_member_distance, p.clustering};
  h = fnv1a(h, v, sizeof(v));
  h = fnv1a(h, p.hash_code_map, sizeof(p.hash_code_map));
  h = fnv1a(h, p.similarity_code_map, sizeof(p.similarity_code_map));
  h = fnv1a(h, p.code_scores, sizeof(p.code_scores));
  return h;
}

// a cheap check that the blob belongs to these residues: offsets, and up to
// 64 KB of codes from each end
inline uint64_t db_check(const uint8_t *codes, uint64_t length, const uint32_t *offsets,
                         uint32_t nseq) {
  uint64_t h = 0xcbf29ce484222325ull;
  h = fnv1a(h, offsets, 4 * ((size_t)nseq + 1));
  const uint64_t k = length < 65536 ? length : 65536;
  h = fnv1a(h, codes, k);
  h = fnv1a(h, codes + length - k, k);
  return h;
}

inline uint64_t pad8(uint64_t n) { return (n + 7) & ~7ull; }

inline void index_array_sizes(const IndexHeader &h, uint64_t n[10]) {
  n[0] = h.n_nc_keys;        // nc_keys
  n[1] = h.n_nc_keys + 1;    // nc_offsets
  n[2] = h.n_nc_values;      // nc_values
  n[3] = h.n_rep_keys;       // rep_keys
  n[4] = h.n_rep_keys + 1;   // rep_offsets
  n[5] = h.n_reps;           // rep_positions
  n[6] = h.n_reps;           // rep_cluster_ids
  n[7] = h.n_reps;           // rep_windows (8 bytes each)
  n[8] = h.n_reps + 1;       // member_offsets
  n[9] = h.n_members;        // member_positions
}

inline uint64_t index_blob_bytes(const IndexHeader &h) {
  uint64_t n[10];
  index_array_sizes(h, n);
  uint64_t b = sizeof(IndexHeader);
  for (int i = 0; i < 10; ++i) b += pad8(n[i] * (i == 7 ? 8 : 4));
  return b;
}

}  // namespace gzb
