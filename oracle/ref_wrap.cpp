/*
 * ref_wrap.cpp -- C entry points over the reference's own arithmetic units.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together
 * with reference sources taken in place from the reference checkout into
 * oracle/_ref/libgzref.so.  Tests use it to pin the C restatement in
 * gz_oracle.c to the reference's behaviour.  Nothing here is shipped.
 */
#include <stdint.h>
#include <string.h>
#include <vector>
#include <string>
#include <sstream>

#include "gz_oracle.h"

#include "alphabet_coder.h"
#include "score_matrix.h"
#include "reduced_alphabet_variable_hash_function.h"
#include "distance_calculator.h"
#include "ungapped_extender.h"
#include "gapped_extender.h"
#include "chain_filter.h"
#include "seed_searcher_database_parameters.h"
#include "statistics.h"
#include "protein_type.h"
#include "sequence.h"
#include "translator.h"
#include "translated_dna_query.h"
#include "sequence_no_filter.h"
#include "sequence_seg_filter.h"
#include "protein_query.h"

static ScoreMatrix make_matrix(const gzo_params *p) {
  std::vector<int> m(p->number_letters * p->number_letters);
  for (int i = 0; i < p->number_letters * p->number_letters; ++i)
    m[i] = p->score_matrix[i];
  return ScoreMatrix("BLOSUM62", &m[0], p->number_letters);
}

/* The reference builds its hash function inside
 * SeedSearcherDatabaseParameters::Build
 * (src/seed_searcher_database_parameters.cpp:52-75); rebuild it the same way. */
static ReducedAlphabetVariableHashFunction make_hash(const gzo_params *p) {
  std::vector<AlphabetCoder::Code> map(p->map_size);
  for (int i = 0; i < p->map_size; ++i) map[i] = p->hash_code_map[i];
  std::vector<int> scores(p->max_indexing_code + 1);
  for (int i = 0; i <= p->max_indexing_code; ++i) scores[i] = p->code_scores[i];
  return ReducedAlphabetVariableHashFunction(
      (AlphabetCoder::Code)p->max_indexing_code, p->seed_threshold,
      p->max_hash_length, map, scores);
}

extern "C" {

int gzr_hash(const gzo_params *p, const uint8_t *seq, uint32_t *hash,
             uint32_t *hash_length) {
  ReducedAlphabetVariableHashFunction f = make_hash(p);
  return f.CalculateHash(seq, hash, hash_length);
}

int gzr_hash_many(const gzo_params *p, const uint8_t *seq, uint32_t n,
                  int32_t *ret, uint32_t *hash, uint32_t *hash_length) {
  ReducedAlphabetVariableHashFunction f = make_hash(p);
  for (uint32_t i = 0; i < n; ++i)
    ret[i] = f.CalculateHash(seq + i, &hash[i], &hash_length[i]);
  return 0;
}

int gzr_distances(const gzo_params *p, const uint8_t *seq0,
                  const uint8_t *seq1, size_t n, uint32_t *c0, uint32_t *c1,
                  int8_t *out) {
  std::vector<AlphabetCoder::Code> map(32);
  for (int i = 0; i < 32; ++i) map[i] = p->similarity_code_map[i];
  DistanceCalculator d;
  d.SetQueries(seq0);
  d.SetDatabase(seq1);
  d.SetReducedCodeMap(&map[0]);
  return d.CalculateDistances(n, c0, c1, p->subsequence_length, (char *)out);
}

int gzr_ungapped_one_side(const gzo_params *p, const uint8_t *seq0,
                          const uint8_t *seq1, int reversed, int cutoff) {
  ScoreMatrix m = make_matrix(p);
  int best = 0;
  UngappedExtender::ExtendOneSideScoreOnly(seq0, seq1, p->delimiter,
                                           reversed != 0, m, cutoff, &best);
  return best;
}

int gzr_gapped_one_side(const gzo_params *p, const uint8_t *seq0,
                        uint32_t seq0_length, const uint8_t *seq1,
                        int reversed, int cutoff, int *best_score,
                        int *best_pos0, int *best_pos1) {
  ScoreMatrix m = make_matrix(p);
  GappedExtender e;
  e.ExtendOneSide(seq0, seq0_length, seq1, p->delimiter, reversed != 0, m,
                  p->gap_open, p->gap_extension, cutoff, best_score,
                  best_pos0, best_pos1, NULL);
  return 0;
}

// GappedExtender::ExtendOneSide with EditBlocks (the traceback the build
// results step uses); ops receive EditBlocks::ToVector().  Returns -1 when
// ops_cap is too small.
int gzr_gapped_one_side_edits(const gzo_params *p, const uint8_t *seq0,
                              uint32_t seq0_length, const uint8_t *seq1,
                              int reversed, int cutoff, int *best_score,
                              int *best_pos0, int *best_pos1, uint8_t *ops,
                              size_t ops_cap, size_t *n_ops) {
  ScoreMatrix m = make_matrix(p);
  GappedExtender e;
  EditBlocks blocks;
  e.ExtendOneSide(seq0, seq0_length, seq1, p->delimiter, reversed != 0, m,
                  p->gap_open, p->gap_extension, cutoff, best_score,
                  best_pos0, best_pos1, &blocks);
  std::vector<EditBlocks::EditOpType> v = blocks.ToVector();
  *n_ops = v.size();
  if (v.size() > ops_cap) return -1;
  for (size_t i = 0; i < v.size(); ++i) ops[i] = (uint8_t)v[i];
  return 0;
}

size_t gzr_chain_filter(const gzo_params *p, const uint8_t *query,
                        uint32_t query_length, int cutoff, const uint8_t *db,
                        uint32_t *hit_q, uint32_t *hit_d, size_t n) {
  ScoreMatrix m = make_matrix(p);
  ChainFilter f(p->delimiter, m);
  std::vector<ChainFilter::Hit> hits(n);
  for (size_t i = 0; i < n; ++i) {
    hits[i].query_sequence_position = hit_q[i];
    hits[i].database_sequence_position = hit_d[i];
    hits[i].k_mer_count = 1;
  }
  f.Filter(query, query_length, cutoff, db, hits);
  for (size_t i = 0; i < hits.size(); ++i) {
    hit_q[i] = hits[i].query_sequence_position;
    hit_d[i] = hits[i].database_sequence_position;
  }
  return hits.size();
}

/* Database index built by the reference builder; looked up key by key. */
struct gzr_db_index {
  SeedSearcherDatabaseParameters params;
  std::vector<AlphabetCoder::Code> seq;
};

void *gzr_db_index_build(const gzo_params *p, const uint8_t *db,
                         uint32_t length) {
  gzr_db_index *x = new gzr_db_index;
  x->seq.assign(db, db + length);
  SeedSearcherDatabaseParameters::BuildParameters bp;
  bp.clustering = p->clustering != 0;
  bp.subsequence_length = p->subsequence_length;
  bp.max_indexing_code = (AlphabetCoder::Code)p->max_indexing_code;
  bp.sequence_delimiter = (AlphabetCoder::Code)p->delimiter;
  bp.seed_threshold = p->seed_threshold;
  bp.threshold = 0.0f;
  bp.number_threads = 1;
  bp.hash_code_map.assign(p->hash_code_map, p->hash_code_map + p->map_size);
  bp.similairty_code_map.assign(p->similarity_code_map,
                                p->similarity_code_map + p->map_size);
  bp.score_matrix = make_matrix(p);
  x->params.Build(&x->seq[0], length, bp);
  return x;
}

void gzr_db_index_free(void *h) { delete (gzr_db_index *)h; }

/* which: 0 residual values, 1 representatives (cluster id, position) */
size_t gzr_db_index_lookup(void *h, int which, uint32_t key, uint32_t *out,
                           size_t cap) {
  gzr_db_index *x = (gzr_db_index *)h;
  if (which == 0) {
    const uint32_t *v = NULL;
    size_t n = 0;
    if (x->params.GetSequencesIndex().GetValues(key, &v, &n)) return 0;
    for (size_t i = 0; i < n && i < cap; ++i) out[i] = v[i];
    return n;
  }
  const SeedSearcherDatabaseParameters::ClusteringSequencesIndex::
      RepresentativeData *r = NULL;
  size_t n = 0;
  if (x->params.GetClusteringSequencesIndex().GetRepresentatives(key, &r, &n))
    return 0;
  for (size_t i = 0; i < n && 2 * i + 1 < cap; ++i) {
    out[2 * i] = r[i].first;
    out[2 * i + 1] = r[i].second;
  }
  return n;
}

size_t gzr_db_index_members(void *h, uint32_t cluster_id, uint32_t *out,
                            size_t cap) {
  gzr_db_index *x = (gzr_db_index *)h;
  const uint32_t *m = NULL;
  size_t n = 0;
  if (x->params.GetClusteringSequencesIndex().GetMembers(cluster_id, &m, &n))
    return 0;
  for (size_t i = 0; i < n && i < cap; ++i) out[i] = m[i];
  return n;
}

int gzr_db_index_max_mismatches(void *h) {
  return ((gzr_db_index *)h)->params.GetNumberMaxMismatchs();
}

/* The index as the reference's `db` command writes it to the chunk's .sdp
 * file (SeedSearcherDatabaseParameters::Save,
 * src/seed_searcher_database_parameters.cpp:363-376); returns its size and
 * copies up to cap bytes. */
/* The database's common parameter file (.scp, SaveCommonParameters,
 * src/seed_searcher_database_parameters.cpp:378-387); as gzr_db_index_save. */
size_t gzr_db_index_save_common(void *h, uint8_t *out, size_t cap) {
  std::ostringstream os(std::ios::binary);
  ((gzr_db_index *)h)->params.SaveCommonParameters(os);
  const std::string b = os.str();
  if (out) memcpy(out, b.data(), b.size() < cap ? b.size() : cap);
  return b.size();
}

size_t gzr_db_index_save(void *h, uint8_t *out, size_t cap) {
  std::ostringstream os(std::ios::binary);
  ((gzr_db_index *)h)->params.Save(os);
  const std::string b = os.str();
  if (out) memcpy(out, b.data(), b.size() < cap ? b.size() : cap);
  return b.size();
}

/* Cutoffs exactly as the reference derives them from bit scores
 * (src/statistics.cpp:28-43, :191-249). */
int gzr_ungapped_karlin(const gzo_params *p, const uint8_t *seq,
                        uint32_t length, float *lambda, float *k, float *h) {
  ProteinType t;
  Statistics s(t);
  ScoreMatrix m = make_matrix(p);
  Statistics::KarlinParameters kp;
  bool ok = s.CalculateUngappedKarlinParameters(seq, length, m, &kp);
  if (!ok) s.CalculateUngappedIdealKarlinParameters(m, &kp);
  *lambda = kp.lambda;
  *k = kp.K;
  *h = kp.H;
  return ok ? 0 : 1;
}

int gzr_normalized_cutoff_to_nominal(float bits, float lambda, float k) {
  Statistics::KarlinParameters kp;
  kp.lambda = lambda;
  kp.K = k;
  kp.H = 0;
  return Statistics::NormalizedCutoff2NominalCutoff(bits, kp);
}

int gzr_normalized_to_nominal(float bits, float lambda, float k) {
  Statistics::KarlinParameters kp;
  kp.lambda = lambda;
  kp.K = k;
  kp.H = 0;
  return Statistics::Normalized2Nominal(bits, kp);
}


/* TranslatedDnaQuery as Queries::BuildQuery makes it for a DNA read with
 * filtering off (src/queries.cpp:83-107, src/translated_dna_query.cpp:27-74);
 * copies the translated codes to out (capacity cap) and returns their
 * number.  Reads shorter than 3 bases are outside what the reference
 * handles and must not be passed. */
uint32_t gzr_translate_query(const gzo_params *p, const char *dna, uint32_t length,
                             uint8_t *out, uint32_t cap) {
  Sequence seq("read", std::string(dna, length));
  Translator translator;
  SequenceNoFilter filter;
  ScoreMatrix m = make_matrix(p);
  ProteinType t;
  Statistics s(t);
  Statistics::KarlinParameters ideal;
  s.CalculateUngappedIdealKarlinParameters(m, &ideal);
  TranslatedDnaQuery q(seq, p->delimiter, translator, &filter, m, ideal);
  Query &base = q;  /* the static GetSequenceLength(uint32_t) hides the virtual one */
  const uint32_t n = base.GetSequenceLength();
  const AlphabetCoder::Code *codes = base.GetSequence();
  for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = codes[i];
  return n;
}


/* SequenceSegFilter::Filter (src/sequence_seg_filter.cpp:17-23) on one
 * protein string: returns its code and, when 0, the masked string in out. */
int gzr_seg_mask(const char *seq, uint32_t length, char *out) {
  SequenceSegFilter filter;
  std::string masked;
  const int rc = filter.Filter(std::string(seq, length), &masked);
  if (rc == 0) memcpy(out, masked.data(), masked.size());
  return rc;
}

/* TranslatedDnaQuery with the SEG filter (Queries::GetFilter with filter
 * on, src/queries.cpp:50-63). */
uint32_t gzr_translate_query_seg(const gzo_params *p, const char *dna, uint32_t length,
                                 uint8_t *out, uint32_t cap) {
  Sequence seq("read", std::string(dna, length));
  Translator translator;
  SequenceSegFilter filter;
  ScoreMatrix m = make_matrix(p);
  ProteinType t;
  Statistics s(t);
  Statistics::KarlinParameters ideal;
  s.CalculateUngappedIdealKarlinParameters(m, &ideal);
  TranslatedDnaQuery q(seq, p->delimiter, translator, &filter, m, ideal);
  Query &base = q;
  const uint32_t n = base.GetSequenceLength();
  const AlphabetCoder::Code *codes = base.GetSequence();
  for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = codes[i];
  return n;
}


/* ProteinQuery with the SEG filter on: copies its length + 2 codes to out
 * and its ungapped Karlin parameters. */
uint32_t gzr_protein_query_seg(const gzo_params *p, const char *letters, uint32_t length,
                               uint8_t *out, uint32_t cap, float *lambda, float *k) {
  Sequence seq("query", std::string(letters, length));
  SequenceSegFilter filter;
  ScoreMatrix m = make_matrix(p);
  ProteinType t;
  Statistics s(t);
  Statistics::KarlinParameters ideal;
  s.CalculateUngappedIdealKarlinParameters(m, &ideal);
  ProteinQuery q(seq, p->delimiter, &filter, m, ideal);
  Query &base = q;
  const uint32_t n = base.GetSequenceLength();
  const AlphabetCoder::Code *codes = base.GetSequence();
  for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = codes[i];
  Statistics::KarlinParameters kp = base.GetUngappedKarlinParameters();
  *lambda = kp.lambda;
  *k = kp.K;
  return n;
}


/* The hit table's statistics as AlignerCommon::WriteOutput takes them
 * (src/aligner_common.h:344-394), for the protein aligner with the score
 * matrix and gaps of p (gapped Karlin parameters and alpha, beta from
 * src/statistics.cpp:232-270). */
int gzr_hit_statistics(const gzo_params *p, uint64_t query_length, uint64_t db_length,
                       uint64_t db_sequences, int32_t score, uint64_t *search_space,
                       double *evalue, float *bit_score) {
  ProteinType t;
  Statistics s(t);
  ScoreMatrix m = make_matrix(p);
  Statistics::KarlinParameters kp;
  double alpha = 0, beta = 0;
  if (!s.CalculateGappedKarlinParameters(m, p->gap_open, p->gap_extension, &kp)) return 1;
  if (!s.CalculateAlphaBeta(m, p->gap_open, p->gap_extension, &alpha, &beta)) return 1;
  *search_space = s.CalculateSearchSpace(query_length, db_length, db_sequences, kp, alpha, beta);
  *evalue = Statistics::Nominal2EValue(score, *search_space, kp);
  *bit_score = Statistics::Nominal2Normalized(score, kp);
  return 0;
}

/* TranslatedDnaQuery::GetRealStart / GetRealEnd of a read's query. */
void gzr_translated_real(const gzo_params *p, const char *dna, uint32_t length,
                         uint32_t position, uint32_t *start, uint32_t *end) {
  Sequence seq("read", std::string(dna, length));
  Translator translator;
  SequenceNoFilter filter;
  ScoreMatrix m = make_matrix(p);
  ProteinType t;
  Statistics s(t);
  Statistics::KarlinParameters ideal;
  s.CalculateUngappedIdealKarlinParameters(m, &ideal);
  TranslatedDnaQuery q(seq, p->delimiter, translator, &filter, m, ideal);
  *start = q.GetRealStart(position);
  *end = q.GetRealEnd(position);
}

} /* extern "C" */
