// gzb_index.cuh -- device layout of the seed index and query hash lists.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ghostz_b200.h"

namespace gzb {

// Device copy of the search parameters the kernels read.
struct DevParams {
  int delimiter;
  int number_letters;
  int map_size;
  int max_indexing_code;
  int seed_threshold;
  int max_hash_length;
  int min_hash_length;
  int subsequence_length;
  int max_member_distance;
  int distance_threshold;
  int shift;
  uint8_t hash_map[32];     // residue code -> reduced code + 1, 0 = unhashable
  uint8_t sim_map[32];
  int code_scores[32];      // indexed by reduced code + 1
};

// Variable-length reduced-alphabet hash
// (ReducedAlphabetVariableHashFunction::CalculateHash,
// src/reduced_alphabet_variable_hash_function.cpp:56-86): returns false when
// one of the first max_hash_length residues examined is not hashable.
__device__ __forceinline__ bool seed_hash(const DevParams &p, const uint8_t *s,
                                          uint32_t *hash, int *hash_length) {
  uint32_t h = 0;
  int score = 0;
  int k;
  for (k = 0; k < p.max_hash_length; ++k) {
    const int c = s[k];
    const int r = c < p.map_size ? p.hash_map[c] : 0;
    if (r == 0) return false;
    if (k >= p.min_hash_length && score >= p.seed_threshold) break;
    h = (h << p.shift) + (uint32_t)r;
    score += p.code_scores[r];
  }
  *hash = h;
  *hash_length = k;
  return true;
}

// Seed index of one database chunk: CSR arrays keyed by hash.
struct DevIndex {
  uint32_t *nc_keys = nullptr, *nc_offsets = nullptr, *nc_values = nullptr;
  uint32_t *rep_keys = nullptr, *rep_offsets = nullptr;
  uint32_t *rep_cluster_ids = nullptr, *rep_positions = nullptr;
  uint32_t *member_offsets = nullptr, *member_positions = nullptr;
  uint64_t *rep_windows = nullptr;  // packed similarity window per representative
  uint64_t n_nc_keys = 0, n_nc_values = 0, n_rep_keys = 0, n_reps = 0,
           n_members = 0;
  bool params_clustering = false;  // built with clustering (rep/member arrays)
};

// Query hash lists (SeedSearcherGpuQueryParameters, seed search inputs).
struct DevLists {
  uint32_t *hash = nullptr;      // per list
  uint32_t *offsets = nullptr;   // per list + 1, into the entry arrays
  uint32_t *nchk = nullptr;      // check positions per list (they come first)
  uint32_t *rep_begin = nullptr, *rep_count = nullptr;  // rep index range
  uint32_t *nc_begin = nullptr, *nc_count = nullptr;    // residual range
  uint64_t *unit_offsets = nullptr;                     // per list + 1
  uint32_t *entry_qid = nullptr;   // per entry: query id
  uint32_t *entry_cpos = nullptr;  // concatenated position
  uint64_t *entry_window = nullptr;  // packed similarity window (check entries)
  uint32_t *entry_ct = nullptr;      // the entry's query cutoff << 16 | (uint16) trigger
  uint64_t n_lists = 0, n_entries = 0, n_units = 0;
};

// Similarity codes of the L-window centred on `center`, 4 bits per code
// (window[t] in bits 4t..4t+3); the distance of two windows is the number
// of differing nibbles (DistanceCalculator::CalculateDistance,
// src/distance_calculator.cpp:35-54).
__device__ __forceinline__ uint64_t pack_window(const DevParams &p, const uint8_t *center) {
  const int L = p.subsequence_length, half = L / 2;
  uint64_t w = 0;
  for (int t = 0; t < L; ++t) {
    const int x = center[t - half];
    w |= (uint64_t)((x < 32 ? p.sim_map[x] : 0) & 15) << (4 * t);
  }
  return w;
}

__device__ __forceinline__ int nibble_mismatches(uint64_t a, uint64_t b) {
  uint64_t x = a ^ b;
  x = (x | (x >> 1) | (x >> 2) | (x >> 3)) & 0x1111111111111111ull;
  return __popcll(x);
}

// Binary search in a sorted key array; returns index or -1.
__device__ __forceinline__ long long find_key(const uint32_t *keys, uint64_t n,
                                              uint32_t key) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (keys[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < n && keys[lo] == key) ? (long long)lo : -1;
}

// Largest i in [lo, hi] with off[i] <= v (off non-decreasing, off[lo] <= v).
__device__ __forceinline__ uint64_t upper_segment(const uint64_t *off, uint64_t lo,
                                                  uint64_t hi, uint64_t v) {
  while (lo < hi) {
    const uint64_t mid = (lo + hi + 1) >> 1;
    if (off[mid] <= v)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

}  // namespace gzb
