// gzb_refindex.cu -- converts the reference's on-disk seed-searcher index of
// one database chunk (the `.sdp` file) into this library's index blob, the
// one gzb_engine_set_database_with_index loads, so a database built by the
// reference's `db` command is searched without an index build.  Host code
// only: no device is touched.
//
// The `.sdp` stream is SeedSearcherDatabaseParameters::Save
// (src/seed_searcher_database_parameters.cpp:363-376), written per chunk by
// DatabaseChunk::SaveSeedSearcherParameters (src/database_chunk.h:461-470):
//   bool clustering, uint8 delimiter, uint32 subsequence length,
//   the residual index (VariableHashSequencesIndex::Save,
//     src/variable_hash_sequences_index.cpp:51-54: hash function, then a
//     DenseHashInvertedIndex<uint32 hash, uint32 position>),
//   the clustering index (VariableHashClusteringSeuencesIndex::Save,
//     src/variable_hash_clustering_seuences_index.cpp:59-63: hash function,
//     DenseHashInvertedIndex<uint32 hash, (uint32 cluster id, uint32
//     position)> of representatives, PerfectHashInvertedIndex<uint32 cluster
//     id, uint32 position> of members),
//   float cluster threshold rate, then the similarity code map.
// Hash function (ReducedAlphabetVariableHashFunction::Save,
// src/reduced_alphabet_variable_hash_function.cpp:133-149): bool, uint8 max
// code, int score threshold, uint32 max length, uint32 shift, uint32 max
// hash, the reduced code map, the code scores.  Dense index
// (src/dense_hash_inverted_index.h:143-159): the (key, key index) pairs of
// its hash map, the offsets by key index, the values.  Perfect index
// (src/perfect_hash_inverted_index.h:125-135): max key, offsets by key,
// values.  Vectors are a 64-bit element count followed by the elements; the
// whole stream is native little-endian, as the reference writes it.

#include <algorithm>
#include <cstring>
#include <utility>
#include <vector>

#include "ghostz_b200.h"
#include "gzb_blob.h"
#include "gzb_common.h"

namespace {

using namespace gzb;

// Sequential reader; a read past the end fails and poisons the reader.
struct Reader {
  const uint8_t *p;
  uint64_t n, at;
  bool ok;
  template <class T>
  bool get(T *v) {
    if (!ok || n - at < sizeof(T)) return ok = false;
    memcpy(v, p + at, sizeof(T));
    at += sizeof(T);
    return true;
  }
  template <class T>
  bool get_vector(std::vector<T> *v) {
    uint64_t k = 0;
    if (!get(&k)) return false;
    if (k > (n - at) / sizeof(T)) return ok = false;
    v->resize(k);
    if (k) memcpy(v->data(), p + at, k * sizeof(T));
    at += k * sizeof(T);
    return true;
  }
};

struct RefHash {
  uint8_t usable = 0, max_code = 0;
  int32_t threshold = 0;
  uint32_t max_length = 0, shift = 0, max_hash = 0;
  std::vector<uint8_t> map;
  std::vector<int32_t> scores;
};

bool read_hash(Reader &r, RefHash *h) {
  return r.get(&h->usable) && r.get(&h->max_code) && r.get(&h->threshold) &&
         r.get(&h->max_length) && r.get(&h->shift) && r.get(&h->max_hash) &&
         r.get_vector(&h->map) && r.get_vector(&h->scores);
}

// DenseHashInvertedIndex: values of key k are values[offsets[i] ..
// offsets[i + 1]) where (k, i) is one of the stored pairs.
template <class V>
struct RefDense {
  std::vector<std::pair<uint32_t, uint32_t>> keys;
  std::vector<uint32_t> offsets;
  std::vector<V> values;
};

template <class V>
bool read_dense(Reader &r, RefDense<V> *d) {
  uint64_t nk = 0;
  if (!r.get(&nk)) return false;
  if (nk > (r.n - r.at) / 8) return r.ok = false;
  d->keys.resize(nk);
  for (auto &kv : d->keys)
    if (!r.get(&kv.first) || !r.get(&kv.second)) return false;
  return r.get_vector(&d->offsets) && r.get_vector(&d->values);
}

// (key, index) pairs sorted by key: two counting passes over 16-bit digits
// (keys are distinct, so the order among equal keys never matters).
void sort_by_key(std::vector<std::pair<uint32_t, uint32_t>> *v) {
  std::vector<std::pair<uint32_t, uint32_t>> tmp(v->size());
  std::vector<uint64_t> count(1 << 16);
  for (int pass = 0; pass < 2; ++pass) {
    const int shift = 16 * pass;
    std::fill(count.begin(), count.end(), 0);
    for (const auto &kv : *v) ++count[(kv.first >> shift) & 0xFFFF];
    uint64_t sum = 0;
    for (auto &c : count) {
      const uint64_t n = c;
      c = sum;
      sum += n;
    }
    for (const auto &kv : *v) tmp[count[(kv.first >> shift) & 0xFFFF]++] = kv;
    v->swap(tmp);
  }
}

// The pairs sorted by key, each key's value range checked; false if the
// index is inconsistent.
template <class V>
bool sorted_ranges(const RefDense<V> &d, std::vector<std::pair<uint32_t, uint32_t>> *out) {
  const uint64_t nk = d.keys.size();
  if (d.offsets.size() != nk + 1 || d.offsets[nk] != d.values.size()) return false;
  for (uint64_t i = 0; i < nk; ++i)
    if (d.offsets[i] > d.offsets[i + 1]) return false;
  *out = d.keys;
  sort_by_key(out);
  std::vector<uint8_t> seen(nk, 0);
  for (uint64_t i = 0; i < nk; ++i) {
    const auto &kv = (*out)[i];
    if (i && kv.first == (*out)[i - 1].first) return false;  // a key twice
    if (kv.second >= nk || seen[kv.second]) return false;    // index not a permutation
    seen[kv.second] = 1;
  }
  return true;
}

// a representative as the file stores it: (cluster id, position)
struct RefRep {
  uint32_t cluster, position;
};

struct RefPerfect {
  uint32_t max_key = 0;
  std::vector<uint32_t> offsets, values;
};

bool read_perfect(Reader &r, RefPerfect *m) {
  return r.get(&m->max_key) && r.get_vector(&m->offsets) && r.get_vector(&m->values);
}

// the similarity window of the device build (pack_window): codes outside the
// chunk read as the delimiter, as the device's padding does
uint64_t host_window(const gzb_params &p, const uint8_t *codes, uint64_t length, uint32_t pos) {
  const int L = p.subsequence_length, half = L / 2;
  uint64_t w = 0;
  for (int t = 0; t < L; ++t) {
    const int64_t i = (int64_t)pos - half + t;
    const int x = (i >= 0 && (uint64_t)i < length) ? codes[i] : p.delimiter;
    w |= (uint64_t)((x < 32 ? p.similarity_code_map[x] : 0) & 15) << (4 * t);
  }
  return w;
}

// The hash function the file was built with must be the one `p` describes
// (SeedSearcherDatabaseParameters::Build makes it from the hash code map,
// the seed threshold, the largest indexing code and max length 8,
// src/seed_searcher_database_parameters.cpp:52-75).  Its constructor keeps
// every reduced code and the largest one plus one, and the code scores
// shifted up by one behind a 0 (code 0 stands for no code,
// src/reduced_alphabet_variable_hash_function.cpp:18-42).
bool hash_matches(const RefHash &h, const gzb_params &p) {
  if (h.max_code != (uint32_t)p.max_indexing_code + 1 || h.threshold != p.seed_threshold ||
      h.max_length != (uint32_t)p.max_hash_length || h.map.size() != (size_t)p.map_size ||
      h.scores.size() != (size_t)p.max_indexing_code + 2 || h.scores[0] != 0)
    return false;
  for (int i = 0; i < p.map_size; ++i)
    if (h.map[i] != (uint8_t)(p.hash_code_map[i] + 1)) return false;
  for (int c = 0; c <= p.max_indexing_code; ++c)
    if (h.scores[c + 1] != p.code_scores[c]) return false;
  return true;
}

}  // namespace

extern "C" int gzb_index_blob_from_reference(const gzb_params *params, const void *sdp,
                                             uint64_t sdp_bytes, const uint8_t *codes,
                                             uint64_t length, const uint32_t *offsets,
                                             uint32_t number_sequences, void *blob,
                                             uint64_t capacity, uint64_t *blob_bytes) {
  GZB_CHECK(params && sdp && codes && offsets && blob_bytes && number_sequences > 0 &&
                length > 0,
            GZB_ERR_INVALID, "null or empty argument");
  GZB_CHECK(length < (1ull << 31), GZB_ERR_OVERFLOW,
            "database chunk of %llu residues exceeds 2^31", (unsigned long long)length);
  const gzb_params &p = *params;
  GZB_CHECK(p.subsequence_length >= 1 && p.subsequence_length <= 16 && p.map_size > 0 &&
                p.map_size <= 32 && p.max_indexing_code >= 0 && p.max_indexing_code < 32 &&
                p.delimiter >= 0 && p.delimiter < 32,
            GZB_ERR_INVALID, "parameters out of range");
  Reader r{(const uint8_t *)sdp, sdp_bytes, 0, true};
  uint8_t clustering = 0, delimiter = 0;
  uint32_t L = 0;
  RefHash seq_hash, clu_hash;
  RefDense<uint32_t> nc;
  RefDense<RefRep> reps;
  RefPerfect members;
  float rate = 0.f;
  std::vector<uint8_t> sim_map;
  r.get(&clustering) && r.get(&delimiter) && r.get(&L) && read_hash(r, &seq_hash) &&
      read_dense(r, &nc) && read_hash(r, &clu_hash) && read_dense(r, &reps) &&
      read_perfect(r, &members) && r.get(&rate) && r.get_vector(&sim_map);
  GZB_CHECK(r.ok && r.at == sdp_bytes, GZB_ERR_INVALID,
            "not a seed-searcher index file (%s at byte %llu of %llu)",
            r.ok ? "trailing bytes" : "stream ends early", (unsigned long long)r.at,
            (unsigned long long)sdp_bytes);
  // built with the parameters this search uses
  const bool clu = p.clustering != 0;
  GZB_CHECK((clustering != 0) == clu && delimiter == (uint32_t)p.delimiter &&
                L == (uint32_t)p.subsequence_length,
            GZB_ERR_INVALID,
            "index file was built with other parameters (clustering %d, delimiter %d, "
            "window %u)",
            (int)clustering, (int)delimiter, L);
  GZB_CHECK(sim_map.size() == (size_t)p.map_size &&
                std::equal(sim_map.begin(), sim_map.end(), p.similarity_code_map),
            GZB_ERR_INVALID, "index file was built with another similarity code map");
  GZB_CHECK(hash_matches(seq_hash, p) && (!clu || hash_matches(clu_hash, p)), GZB_ERR_INVALID,
            "index file was built with another seed hash");
  if (clu)  // SeedSearcherDatabaseParameters::GetNumberMaxMismatchs, :409-411
    GZB_CHECK((int)((float)L * (1 - rate)) == p.max_member_distance, GZB_ERR_INVALID,
              "index file was built with another cluster threshold (%g)", (double)rate);

  std::vector<std::pair<uint32_t, uint32_t>> nc_keys, rep_keys;
  GZB_CHECK(sorted_ranges(nc, &nc_keys), GZB_ERR_INVALID, "residual index is inconsistent");
  for (uint32_t v : nc.values)
    GZB_CHECK(v < length, GZB_ERR_INVALID, "residual position %u outside the chunk", v);
  if (clu) {
    GZB_CHECK(sorted_ranges(reps, &rep_keys), GZB_ERR_INVALID,
              "representative index is inconsistent");
    const std::vector<uint32_t> &mo = members.offsets;
    GZB_CHECK(mo.size() == (size_t)members.max_key + 2 && mo.back() == members.values.size(),
              GZB_ERR_INVALID, "member index is inconsistent");
    for (size_t i = 0; i + 1 < mo.size(); ++i)
      GZB_CHECK(mo[i] <= mo[i + 1], GZB_ERR_INVALID, "member index is inconsistent");
    for (uint32_t v : members.values)
      GZB_CHECK(v < length, GZB_ERR_INVALID, "member position %u outside the chunk", v);
    for (const auto &cp : reps.values)
      GZB_CHECK(cp.position < length, GZB_ERR_INVALID,
                "representative position %u outside the chunk", cp.position);
  }

  // the blob: keys ascending, each key's values in the file's order; cluster
  // c of this blob is the c-th representative, its members in the file's order
  IndexHeader h;
  memset(&h, 0, sizeof(h));
  h.magic = kIndexMagic;
  h.fingerprint = params_fingerprint(p);
  h.db_len = length;
  h.nseq = number_sequences;
  h.db_check = db_check(codes, length, offsets, number_sequences);
  h.n_nc_keys = nc_keys.size();
  h.n_nc_values = nc.values.size();
  uint64_t n_members = 0;
  if (clu) {
    h.n_rep_keys = rep_keys.size();
    h.n_reps = reps.values.size();
    for (const auto &cp : reps.values)
      if (cp.cluster <= members.max_key)
        n_members += members.offsets[cp.cluster + 1] - members.offsets[cp.cluster];
    h.n_members = n_members;
  }
  GZB_CHECK(h.n_nc_values < (1ull << 32) && h.n_reps < (1ull << 32) && n_members < (1ull << 32),
            GZB_ERR_OVERFLOW, "index too large for 32-bit offsets");
  const uint64_t need = index_blob_bytes(h);
  *blob_bytes = need;
  if (!blob) return GZB_OK;
  GZB_CHECK(capacity >= need, GZB_ERR_INVALID, "index blob needs %llu bytes",
            (unsigned long long)need);
  uint8_t *out = (uint8_t *)blob;
  memset(out, 0, need);
  memcpy(out, &h, sizeof(h));
  uint64_t n[10], at[10], pos = sizeof(h);
  index_array_sizes(h, n);
  for (int i = 0; i < 10; ++i) {
    at[i] = pos;
    pos += pad8(n[i] * (i == 7 ? 8 : 4));
  }
  auto u32 = [&](int a) { return reinterpret_cast<uint32_t *>(out + at[a]); };
  // residual index
  {
    uint32_t *keys = u32(0), *offs = u32(1), *vals = u32(2);
    uint32_t k = 0;
    offs[0] = 0;
    for (const auto &kv : nc_keys) {
      const uint32_t b = nc.offsets[kv.second], e = nc.offsets[kv.second + 1];
      keys[k] = kv.first;
      std::copy(nc.values.begin() + b, nc.values.begin() + e, vals + offs[k]);
      offs[k + 1] = offs[k] + (e - b);
      ++k;
    }
  }
  // representatives and their clusters
  if (clu) {
    uint32_t *keys = u32(3), *offs = u32(4), *rpos = u32(5), *cids = u32(6);
    uint64_t *wins = reinterpret_cast<uint64_t *>(out + at[7]);
    uint32_t *moffs = u32(8), *mpos = u32(9);
    uint32_t k = 0, rep = 0, m = 0;
    offs[0] = 0;
    moffs[0] = 0;
    for (const auto &kv : rep_keys) {
      const uint32_t b = reps.offsets[kv.second], e = reps.offsets[kv.second + 1];
      keys[k] = kv.first;
      for (uint32_t i = b; i < e; ++i, ++rep) {
        const uint32_t cid = reps.values[i].cluster, at_pos = reps.values[i].position;
        rpos[rep] = at_pos;
        cids[rep] = rep;
        wins[rep] = host_window(p, codes, length, at_pos);
        if (cid <= members.max_key) {
          const uint32_t mb = members.offsets[cid], me = members.offsets[cid + 1];
          std::copy(members.values.begin() + mb, members.values.begin() + me, mpos + m);
          m += me - mb;
        }
        moffs[rep + 1] = m;
      }
      offs[k + 1] = offs[k] + (e - b);
      ++k;
    }
  } else {
    u32(4)[0] = 0;
    u32(8)[0] = 0;
  }
  return GZB_OK;
}

// The `.scp` file of a chunk (SeedSearcherDatabaseParameters::
// SaveCommonParameters, src/seed_searcher_database_parameters.cpp:378-387,
// written by DatabaseChunk::SaveSeedSearcherCommonParameters,
// src/database_chunk.h:449-458): uint8 delimiter, uint32 subsequence
// length, the similarity code map, the hash function.
extern "C" int gzb_params_from_reference_common(const void *scp, uint64_t scp_bytes,
                                                gzb_params *params) {
  GZB_CHECK(scp && params, GZB_ERR_INVALID, "null argument");
  Reader r{(const uint8_t *)scp, scp_bytes, 0, true};
  uint8_t delimiter = 0;
  uint32_t L = 0;
  std::vector<uint8_t> sim_map;
  RefHash h;
  r.get(&delimiter) && r.get(&L) && r.get_vector(&sim_map) && read_hash(r, &h);
  GZB_CHECK(r.ok && r.at == scp_bytes, GZB_ERR_INVALID,
            "not a seed-searcher common parameter file (%s at byte %llu of %llu)",
            r.ok ? "trailing bytes" : "stream ends early", (unsigned long long)r.at,
            (unsigned long long)scp_bytes);
  GZB_CHECK(delimiter < 32 && L >= 1 && L <= 16 && !sim_map.empty() && sim_map.size() <= 32 &&
                h.map.size() == sim_map.size() && h.max_code >= 1 && h.max_code <= 32 &&
                h.scores.size() == (size_t)h.max_code + 1 && h.scores[0] == 0 &&
                h.max_length >= 1 && h.max_length <= 16,
            GZB_ERR_INVALID, "common parameter file out of range");
  for (uint8_t c : h.map)
    GZB_CHECK(c >= 1, GZB_ERR_INVALID, "hash code map entry 0 (codes are stored plus one)");
  gzb_params &p = *params;
  p.delimiter = delimiter;
  p.subsequence_length = (int32_t)L;
  p.map_size = (int32_t)sim_map.size();
  memset(p.similarity_code_map, 0, sizeof(p.similarity_code_map));
  memset(p.hash_code_map, 0, sizeof(p.hash_code_map));
  memset(p.code_scores, 0, sizeof(p.code_scores));
  for (size_t i = 0; i < sim_map.size(); ++i) {
    p.similarity_code_map[i] = sim_map[i];
    p.hash_code_map[i] = (uint8_t)(h.map[i] - 1);
  }
  p.max_indexing_code = h.max_code - 1;
  for (int c = 0; c + 1 < (int)h.scores.size(); ++c) p.code_scores[c] = h.scores[c + 1];
  p.seed_threshold = h.threshold;
  p.max_hash_length = (int32_t)h.max_length;
  return GZB_OK;
}
