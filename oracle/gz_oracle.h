/*
 * gz_oracle.h -- CPU restatement of the GHOSTZ-GPU presearch path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * engine is compared against.  Only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load it; the engine never does.
 *
 * Every function restates one reference function (file:line given at the
 * definition in gz_oracle.c) in plain C, sequentially, with no GPU code.
 * Parity with the reference itself is pinned by tests that run the
 * reference's own sources (compiled by oracle/Makefile into oracle/_ref)
 * and by the known-answer vectors of the reference's unit tests.
 */
#ifndef GZ_ORACLE_H_
#define GZ_ORACLE_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Search parameters shared by every stage.  Layout is plain int32/uint8
 * so the Python side can fill it with a numpy structured array. */
typedef struct {
  int32_t delimiter;             /* sequence delimiter code (25 for protein) */
  int32_t number_letters;        /* score matrix is number_letters^2 (<= 32) */
  int32_t score_matrix[32 * 32]; /* [db_code * number_letters + query_code] */
  int32_t map_size;              /* entries used in the two code maps (<= 32) */
  uint8_t hash_code_map[32];     /* residue code -> hash (reduced) code */
  uint8_t similarity_code_map[32]; /* residue code -> similarity code */
  int32_t max_indexing_code;     /* largest reduced code that may be hashed */
  int32_t code_scores[32];       /* per reduced code: max self score */
  int32_t seed_threshold;        /* stop hashing once score sum >= this (39) */
  int32_t max_hash_length;       /* 8 */
  int32_t min_hash_length;       /* 6 */
  int32_t subsequence_length;    /* clustering / distance window L (10) */
  int32_t max_member_distance;   /* L * (1 - 0.9f), truncated */
  int32_t distance_threshold;    /* L - 0.8f * L, truncated */
  int32_t gap_open;
  int32_t gap_extension;
  int32_t gapped_cutoff;         /* X-drop of the gapped extension (nominal) */
  int32_t max_number_results;    /* -b */
  int32_t max_number_one_subject_results; /* -v */
  int32_t clustering;            /* 1 when the database was built with -C T */
  int32_t result_gapped_cutoff;  /* X-drop of the build results traceback */
} gzo_params;

/* ---- stage primitives ------------------------------------------------ */
int gzo_hash(const gzo_params *p, const uint8_t *seq, uint32_t *hash,
             uint32_t *hash_length);
int gzo_distance(const gzo_params *p, const uint8_t *seq0,
                 uint32_t center0, const uint8_t *seq1, uint32_t center1);
int gzo_ungapped_one_side(const gzo_params *p, const uint8_t *seq0,
                          const uint8_t *seq1, int reversed, int cutoff);
int gzo_ungapped_with_trigger(const gzo_params *p, const uint8_t *query,
                              uint32_t query_position, const uint8_t *db,
                              uint32_t db_position, int cutoff, int trigger);
/* Score-only affine X-drop extension from seq0[0]/seq1[0] (query/db).
 * best positions are offsets in sequence coordinates (negative when
 * reversed); *cells receives the number of DP cells evaluated. */
int gzo_gapped_one_side(const gzo_params *p, const uint8_t *seq0,
                        const uint8_t *seq1, int reversed, int cutoff,
                        int *best_score, int *best_pos0, int *best_pos1,
                        uint64_t *cells);
/* Affine X-drop extension with its edit path
 * (GappedExtender::ExtendOneSide with EditBlocks, src/gapped_extender.cpp:70-304,
 * and PickOptimalPath, :473-531).  Same score and positions as
 * gzo_gapped_one_side; ops[0..*n_ops) receives the path expanded one op per
 * aligned column in EditBlocks order (EditBlocks::ToVector,
 * src/edit_blocks.cpp): GZO_OP_GAP0 (gap in seq0: a seq1 residue alone),
 * GZO_OP_SUB, GZO_OP_GAP1.  Returns -1 when ops_cap is too small. */
#define GZO_OP_GAP0 0
#define GZO_OP_SUB 1
#define GZO_OP_GAP1 2
int gzo_gapped_one_side_edits(const gzo_params *p, const uint8_t *seq0,
                              const uint8_t *seq1, int reversed, int cutoff,
                              int *best_score, int *best_pos0, int *best_pos1,
                              uint8_t *ops, size_t ops_cap, size_t *n_ops);
/* Alignment statistics of one presearch result, as
 * AlignerCommon::BuildResult computes them (src/aligner_common.h:275-340)
 * after AlignerBuildResultsThread::Run (src/aligner_build_results_thread.h:
 * 110-160) joined the reversed reverse-side path and the forward path.
 * query / db: the concatenated sequences; hit_q is the hit's position in
 * the concatenated query buffer, hit_d in the chunk.  Returns -1 when a
 * side's path does not fit the scratch. */
typedef struct {
  int32_t score;
  uint32_t start_q, start_d, end_q, end_d;  /* concatenated coordinates */
  uint32_t alignment_length, mismatches, gap_openings, gap_extensions;
} gzo_alignment;
int gzo_build_alignment(const gzo_params *p, const uint8_t *query, uint32_t hit_q,
                        const uint8_t *db, uint32_t hit_d, gzo_alignment *out);
/* Chain filter over the hits of one query.  q/d are in place; returns the
 * number of hits kept (sorted by database position, ties by query pos). */
size_t gzo_chain_filter(const gzo_params *p, const uint8_t *query,
                        uint32_t query_length, int cutoff, const uint8_t *db,
                        uint32_t *hit_q, uint32_t *hit_d, size_t n);

/* ---- database index -------------------------------------------------- */
typedef struct gzo_db_index gzo_db_index;
gzo_db_index *gzo_db_index_build(const gzo_params *p, const uint8_t *db,
                                 uint32_t length);
void gzo_db_index_free(gzo_db_index *x);
/* Array access: which = 0 nc_keys, 1 nc_offsets, 2 nc_values,
 * 3 rep_keys, 4 rep_offsets, 5 rep_cluster_ids, 6 rep_positions,
 * 7 member_offsets, 8 member_positions.  Returns the element count. */
size_t gzo_db_index_array(const gzo_db_index *x, int which,
                          const uint32_t **data);

/* ---- query hash lists ------------------------------------------------ */
typedef struct gzo_query_lists gzo_query_lists;
/* queries: concatenated [delim q0 delim q1 ... delim]; offsets[i] is the
 * leading delimiter of query i; lengths[i] = residues + 2 (both
 * delimiters). */
gzo_query_lists *gzo_query_lists_build(const gzo_params *p,
                                       const uint8_t *queries,
                                       const uint32_t *offsets,
                                       const uint32_t *lengths,
                                       uint32_t number_queries);
void gzo_query_lists_free(gzo_query_lists *x);
/* which = 0 hashes, 1 offsets (n+1), 2 check_counts, 3 query_ids,
 * 4 positions (within query) */
size_t gzo_query_lists_array(const gzo_query_lists *x, int which,
                             const uint32_t **data);

/* ---- full presearch of one database chunk ---------------------------- */
typedef struct {
  int32_t chunk_id;
  int32_t subject_id;
  int32_t score;
  uint32_t hit_q, hit_d;
  uint32_t start_q, start_d;
  uint32_t end_q, end_d;
} gzo_result;

typedef struct {
  uint64_t distance_seeds;     /* representative x check-position pairs */
  uint64_t ungapped_seeds;     /* ungapped extensions run */
  uint64_t ungapped_hits;      /* survivors (score > trigger) */
  uint64_t chained_hits;       /* survivors of the chain filter */
  uint64_t gapped_extensions;  /* one-side extensions (2 per hit) */
  uint64_t gapped_cells;       /* DP cells, counted as in gzo_gapped_one_side */
} gzo_counters;

typedef struct gzo_presearch gzo_presearch;
/* Runs seed search -> distance filter -> ungapped X-drop with trigger ->
 * chain filter -> gapped X-drop (both sides) -> top-b merge for every
 * query against one database chunk.  db_offsets has number_sequences+1
 * entries (first residue of each sequence; last = chunk length).
 * Queries with query_begin <= id < query_end are processed (the others get
 * empty lists); pass 0, number_queries for all. */
gzo_presearch *gzo_presearch_run(const gzo_params *p,
                                 const gzo_db_index *index,
                                 const gzo_query_lists *lists,
                                 const uint8_t *queries,
                                 const uint32_t *query_offsets,
                                 const uint32_t *query_lengths,
                                 uint32_t number_queries,
                                 const int32_t *ungapped_cutoffs,
                                 const int32_t *gapped_triggers,
                                 const uint8_t *db, uint32_t db_length,
                                 const uint32_t *db_offsets,
                                 uint32_t number_sequences,
                                 uint32_t query_begin, uint32_t query_end);
void gzo_presearch_free(gzo_presearch *x);
size_t gzo_presearch_results(const gzo_presearch *x, uint32_t query_id,
                             const gzo_result **results);
void gzo_presearch_counters(const gzo_presearch *x, gzo_counters *out);
/* Ungapped survivors (before chain filtering), sorted by (query, d, q). */
size_t gzo_presearch_hits(const gzo_presearch *x, const uint32_t **qid,
                          const uint32_t **q, const uint32_t **d);

/* Top-b merge of freshly extended results into a running list, as the
 * reference does after each batch of gapped extensions. */
size_t gzo_add_results(const gzo_params *p, const uint32_t *db_offsets,
                       uint32_t number_sequences, uint32_t db_length,
                       gzo_result *added, size_t n_added,
                       gzo_result *results, size_t n_results);


/* Six-frame translation of one DNA read into the reference's translated
 * query layout (TranslatedDnaQuery::SetEncodedSequence,
 * src/translated_dna_query.cpp:44-74, with Translator::Translate,
 * src/translator.cpp:104-142, and no filter): a leading delimiter, then
 * per frame (forward offsets 0,1,2, then the reverse complement's 0,1,2)
 * its codons as protein codes, an extra delimiter when the frame has fewer
 * than length/3 codons, and one closing delimiter.  Returns the bytes
 * written: gzo_translated_length(length).  A read shorter than 3 bases
 * gives [delimiter][delimiter] (the reference writes past an empty buffer
 * for those). */
uint32_t gzo_translated_length(uint32_t length);
uint32_t gzo_translate_query(const char *dna, uint32_t length, uint8_t delimiter,
                             uint8_t *out);


/* Ungapped Karlin-Altschul parameters of one query against the Robinson
 * background and the integer cutoffs derived from them
 * (Statistics::CalculateUngappedKarlinParameters, src/statistics.cpp:205-229,
 * with ext/karlin/src/karlin.c BlastKarlinBlkCalc; cutoffs
 * src/statistics.cpp:28-43 as used at src/aligner_gpu.cpp:228-238).  seq
 * is the whole query, delimiters included; returns 0. */
int gzo_query_karlin(const gzo_params *p, const uint8_t *seq, uint32_t length,
                     float ungapped_bits, float trigger_bits, float *lambda, float *k,
                     float *h, int32_t *cutoff, int32_t *trigger);


/* SEG low-complexity masking of one protein string with window 12
 * (seg::Seg::MaskSequence, ext/seg/src/seg.cpp:98-112, as
 * SequenceSegFilter uses it, src/sequence_seg_filter.cpp:12-23).  Writes
 * the masked string (letters upper-cased, masked residues 'x') to out and
 * returns 0, or returns 1 without writing when the string is shorter than
 * the window. */
int gzo_seg_mask(const char *seq, uint32_t length, char *out);
/* gzo_translate_query with the SEG filter on (Queries::GetFilter,
 * src/queries.cpp:50-63): each frame is masked, and a frame shorter than
 * the window becomes unknown codes (src/translated_dna_query.cpp:59-65). */
uint32_t gzo_translate_query_seg(const char *dna, uint32_t length, uint8_t delimiter,
                                 uint8_t *out);
/* ln(n!) rounded to 6 decimals, as the SEG tables hold it; n <= 65535. */
double gzo_ln_factorial6(uint32_t n);


/* ProteinQuery's codes with the SEG filter on
 * (ProteinQuery::SetEncodedSequence, src/protein_query.cpp:39-49): length + 2
 * codes, [delimiter] masked body [delimiter]; a protein shorter than the
 * window keeps the zero-filled buffer behind the leading delimiter (body
 * and last code 0). */
void gzo_protein_query_seg(const char *letters, uint32_t length, uint8_t delimiter,
                           uint8_t *out);


/* Statistics of the final hit table (AlignerCommon::WriteOutput,
 * src/aligner_common.h:344-394): the search space of a query
 * (Statistics::CalculateSearchSpace with the protein length adjustment,
 * src/statistics.cpp:50-122), E-value (Nominal2EValue, :44-48) and
 * normalized score (Nominal2Normalized, :23-27) under gapped Karlin
 * parameters lambda, k and length-adjustment alpha, beta. */
uint64_t gzo_search_space(uint64_t query_length, uint64_t db_length, uint64_t db_sequences,
                          float lambda, float k, double alpha, double beta);
double gzo_evalue(int32_t score, uint64_t search_space, float lambda, float k);
float gzo_bit_score(int32_t score, float lambda, float k);
/* Read coordinates of a translated query position
 * (TranslatedDnaQuery::GetRealStart / GetRealEnd,
 * src/translated_dna_query.h:43-61). */
uint32_t gzo_translated_real_start(uint32_t position, uint32_t dna_length);
uint32_t gzo_translated_real_end(uint32_t position, uint32_t dna_length);

#ifdef __cplusplus
}
#endif
#endif
