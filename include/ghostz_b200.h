/*
 * ghostz_b200.h -- C ABI of the B200 presearch engine (libghostz_b200.so).
 *
 * The engine replaces the GPU operators of GHOSTZ-GPU's `aln` presearch:
 * seed search over the clustered reduced-alphabet hash index, distance
 * filtering, ungapped X-drop extension with trigger and gapped affine X-drop
 * extension.  Two layers are exported:
 *
 *  1. Per-operator handles whose functions mirror, one to one, the methods of
 *     the reference classes DistanceCalculatorGpu, UngappedExtenderGpu and
 *     GappedExtenderGpu (argument order, meaning, host/device split).  Device
 *     sequences are one byte per residue code (the reference uses a 5-bit
 *     packed form); score matrices use the reference's device layout,
 *     (number_letters + 1)^2 int32 with a zero delimiter row and column
 *     (src/aligner_gpu_data.cu:108-122).
 *  2. A presearch engine that keeps a database chunk, its index and the
 *     queries resident in HBM and runs the whole seed -> ungapped -> chain
 *     filter -> gapped -> top-b pipeline on the device
 *     (the work of AlignerGpuPresearchThread::Run,
 *     src/aligner_gpu_presearch_thread.cpp:62-642).
 *
 * All functions return GZB_OK or an error code (never exit); the message of
 * the last failure on the calling thread is available from gzb_last_error().
 * Handles are not shared between threads without external locking; several
 * handles may use one device concurrently on different streams.
 * `stream` arguments are cudaStream_t passed as void*.
 */
#ifndef GHOSTZ_B200_H_
#define GHOSTZ_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GZB_OK 0
#define GZB_ERR_INVALID 1   /* bad argument or state */
#define GZB_ERR_CUDA 2      /* a CUDA runtime call failed */
#define GZB_ERR_NOMEM 3     /* device or host allocation failed */
#define GZB_ERR_OVERFLOW 4  /* a size exceeds a documented limit */
#define GZB_ERR_TIMEOUT 5   /* a bounded device wait ran out */

const char *gzb_error_string(int code);
const char *gzb_last_error(void);
int gzb_version(void);

/* Search parameters (plain layout; 4-byte fields and byte arrays). */
typedef struct {
  int32_t delimiter;             /* sequence delimiter code (25 for protein) */
  int32_t number_letters;        /* score matrix side (<= 31) */
  int32_t score_matrix[32 * 32]; /* [db_code * number_letters + query_code] */
  int32_t map_size;              /* entries used in the code maps (<= 32) */
  uint8_t hash_code_map[32];     /* residue code -> seed-hash reduced code */
  uint8_t similarity_code_map[32]; /* residue code -> similarity code */
  int32_t max_indexing_code;     /* largest hashable reduced code */
  int32_t code_scores[32];       /* per reduced code: max self score */
  int32_t seed_threshold;        /* hash stops once code scores sum >= this */
  int32_t max_hash_length;       /* 8 */
  int32_t min_hash_length;       /* 6 */
  int32_t subsequence_length;    /* distance / clustering window L */
  int32_t max_member_distance;   /* L * (1 - 0.9f), truncated */
  int32_t distance_threshold;    /* L - 0.8f * L, truncated */
  int32_t gap_open;
  int32_t gap_extension;
  int32_t gapped_cutoff;         /* X-drop of the gapped extension */
  int32_t max_number_results;    /* top-b per query (-b) */
  int32_t max_number_one_subject_results; /* per subject (-v) */
  int32_t clustering;            /* database built with -C T */
  int32_t result_gapped_cutoff;  /* X-drop of the build results step's
                                    traceback (25 normalized bits against 15
                                    for the presearch, src/align_main.cpp:124-125,
                                    src/aligner_gpu.cpp:254-256) */
} gzb_params;

/* Device sequence buffers given to the operators below hold one residue
 * code (< 32) per byte, sequences separated by the delimiter, with at least
 * 64 delimiter bytes before the first and after the last sequence: the
 * kernels read aligned 32-bit words, a few bytes past a delimiter. */

/* ---- DistanceCalculatorGpu (src/distance_calculator_gpu.h:18-40) ------- */
typedef struct gzb_distance_calculator gzb_distance_calculator;
int gzb_distance_calculator_create(gzb_distance_calculator **out);
int gzb_distance_calculator_destroy(gzb_distance_calculator *h);
/* SetQueries / SetDatabase / SetReducedCodeMap / SetSubsequenceLength
 * (src/distance_calculator_gpu.cu:299-318) */
int gzb_distance_calculator_set_queries(gzb_distance_calculator *h,
                                        const uint8_t *d_query_sequence);
int gzb_distance_calculator_set_database(gzb_distance_calculator *h,
                                         const uint8_t *d_database_sequence);
int gzb_distance_calculator_set_reduced_code_map(
    gzb_distance_calculator *h, const uint8_t *d_reduced_code_map);
int gzb_distance_calculator_set_subsequence_length(gzb_distance_calculator *h,
                                                   uint32_t length);
/* CalculateDistancesAsync (src/distance_calculator_gpu.cu:320-355): copies
 * the centres to the device, computes one int8 distance per seed and copies
 * them back, all on `stream`. */
int gzb_distance_calculator_calculate_distances_async(
    gzb_distance_calculator *h, size_t size,
    const uint32_t *query_concatenated_centers,
    const uint32_t *database_centers, int8_t *distances,
    uint32_t *d_query_concatenated_centers, uint32_t *d_database_centers,
    int8_t *d_distances, void *stream);

/* ---- UngappedExtenderGpu (src/ungapped_extender_gpu.h:21-76) ----------- */
typedef struct gzb_ungapped_extender gzb_ungapped_extender;
int gzb_ungapped_extender_create(gzb_ungapped_extender **out);
int gzb_ungapped_extender_destroy(gzb_ungapped_extender *h);
/* SetQuerySeedDataList (src/ungapped_extender_gpu.cu:789-794) */
int gzb_ungapped_extender_set_query_seed_data_list(
    gzb_ungapped_extender *h, const uint32_t *d_query_ids,
    const uint32_t *d_query_positions);
/* SetQueries (src/ungapped_extender_gpu.cu:796-804) */
int gzb_ungapped_extender_set_queries(gzb_ungapped_extender *h,
                                      uint8_t sequence_delimiter,
                                      const uint8_t *d_query_sequence,
                                      const int32_t *d_ungapped_cutoffs,
                                      const int32_t *d_gapped_triggers);
int gzb_ungapped_extender_set_database(gzb_ungapped_extender *h,
                                      const uint8_t *d_database_sequence);
/* SetScoreMatrix (src/ungapped_extender_gpu.cu:811-816) */
int gzb_ungapped_extender_set_score_matrix(gzb_ungapped_extender *h,
                                           const int32_t *d_score_matrix,
                                           uint32_t number_letters);
/* Scratch bytes SetQuerySeeds needs in d_temp_storage for `size` seeds
 * (the reference sizes a CUB scan, src/device_seeds_memory.cu:20-36). */
size_t gzb_ungapped_extender_query_seeds_temp_bytes(size_t size);
/* SetQuerySeeds (src/ungapped_extender_gpu.cu:818-852): expands run-length
 * (query seed id, first seed index) pairs into per-seed query id and
 * concatenated query position. */
int gzb_ungapped_extender_set_query_seeds(
    gzb_ungapped_extender *h, size_t query_seeds_size, size_t size,
    const uint32_t *query_seed_ids, const uint32_t *query_seed_starts,
    size_t temp_storage_bytes, void *d_temp_storage,
    uint32_t *d_query_seed_ids, uint32_t *d_query_seed_starts,
    uint32_t *d_query_ids, uint32_t *d_query_concatenated_positions,
    uint32_t *temp_array, void *stream);
/* ExtendWithTriggerAsync (src/ungapped_extender_gpu.cu:854-899): reverse
 * X-drop from (q-1, d-1), forward from (q, d) while the sum is not above the
 * query's trigger; flags[i] = 1 when the sum exceeds the trigger.  NULL host
 * query ids / positions skip their upload (the device copies are reused). */
int gzb_ungapped_extender_extend_with_trigger_async(
    gzb_ungapped_extender *h, size_t size, const uint32_t *query_ids,
    const uint32_t *query_concatenated_positions,
    const uint32_t *database_positions, int8_t *flags, uint32_t *d_query_ids,
    uint32_t *d_query_concatenated_positions, uint32_t *d_database_positions,
    int8_t *d_flags, int32_t *d_temp_array, void *stream);

/* ---- GappedExtenderGpu (src/gapped_extender_gpu.h:19-60) --------------- */
typedef struct gzb_gapped_extender gzb_gapped_extender;
int gzb_gapped_extender_create(gzb_gapped_extender **out);
int gzb_gapped_extender_destroy(gzb_gapped_extender *h);
/* SetQueries / SetDatabase / SetScoreParameters
 * (src/gapped_extender_gpu.cu:748-767) */
int gzb_gapped_extender_set_queries(gzb_gapped_extender *h,
                                    uint8_t sequence_delimiter,
                                    const uint8_t *d_query_sequence);
int gzb_gapped_extender_set_database(gzb_gapped_extender *h,
                                     const uint8_t *d_database_sequence);
int gzb_gapped_extender_set_score_parameters(gzb_gapped_extender *h,
                                             const int32_t *d_score_matrix,
                                             uint32_t number_letters,
                                             int gap_open, int gap_extension,
                                             int cutoff);
/* ConvertToGappedExtensionSeedsAsync (src/gapped_extender_gpu.cu:769-800):
 * d_out[i] = positions[seed_positions[i]] for query and database
 * positions, the host arrays being uploaded first. */
int gzb_gapped_extender_convert_to_gapped_extension_seeds_async(
    gzb_gapped_extender *h, size_t size, int reverse,
    const uint32_t *seed_positions,
    const uint32_t *query_concatenated_positions,
    const uint32_t *database_positions, uint32_t *d_seed_positions,
    uint32_t *d_temp_array, uint32_t *d_query_concatenated_positions,
    uint32_t *d_database_positions, void *stream);
/* ExtendOneSideScoreOnlyAsync (src/gapped_extender_gpu.cu:802-853): one
 * score-only affine X-drop extension per seed from the device positions
 * (query = sequence0, database = sequence1), forward or reverse.  Positions
 * are replaced by the absolute positions of the best cell; positions and
 * scores are copied back to the host arrays.  Bit-identical to the CPU
 * GappedExtender::ExtendOneSideScoreOnly (src/gapped_extender.cpp:306-471)
 * for every query length (no 128-residue limit). */
int gzb_gapped_extender_extend_one_side_score_only_async(
    gzb_gapped_extender *h, size_t size, int reverse,
    uint32_t *query_concatenated_positions, uint32_t *database_positions,
    int32_t *scores, uint32_t *d_query_concatenated_positions,
    uint32_t *d_database_positions, int32_t *d_scores, void *stream);
/* DP cells evaluated by this handle's extensions so far (synchronous). */
int gzb_gapped_extender_cells(gzb_gapped_extender *h, uint64_t *cells);

/* Gapped one-side extension that allocates no device memory.  No
 * counterpart in the reference: it is the same computation as
 * gzb_gapped_extender_extend_one_side_score_only_async (device buffers only,
 * positions updated in place, scores written; no host copies) for callers
 * that cannot call cudaMalloc themselves -- code running under a host runtime
 * that owns all device memory through its own pool, or a latency-critical
 * loop that cannot take an allocation's implicit device synchronisation.
 * Its scratch is one fixed device array in the library (about 12 MB, held on
 * every GPU that loads the library until exit).  Limits: at most 2^20
 * extensions per call (more: GZB_ERR_OVERFLOW before any device work), and
 * extensions needing the serial fallback may use bands of at most 8192
 * columns (wider: GZB_ERR_OVERFLOW after the kernels have run, the position
 * and score buffers then undefined, so a caller that wants to retry keeps
 * its own copy of the input positions).  Every call shares that array:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * The first call on a device looks up the array's device address (a
 * one-time set-up per device), so make that first call before any stream
 * capture.  Every call ends by reading a counter into host memory and
 * synchronising `stream`. */
int gzb_gapped_extend_one_side_score_only_noalloc(
    const uint8_t *d_query_sequence, const uint8_t *d_database_sequence,
    uint8_t sequence_delimiter, const int32_t *d_score_matrix,
    uint32_t number_letters, int gap_open, int gap_extension, int cutoff,
    size_t size, int reverse, uint32_t *d_query_concatenated_positions,
    uint32_t *d_database_positions, int32_t *d_scores, void *stream);

/* ---- presearch engine ---------------------------------------------------
 * Replaces the device side of AlignerGpuPresearchThread::Run for one
 * database chunk: the seed search of SeedSearcherGpu
 * (src/seed_searcher_gpu.cpp:186-537) with the query lists of
 * SeedSearcherGpuQueryParameters::Build
 * (src/seed_searcher_gpu_query_parameters.cpp:17-272), distance filtering,
 * ungapped extension with trigger, the chain filter
 * (src/chain_filter.cpp:24-99), both gapped extensions and the top-b merge
 * AlignerCommon::AddResults (src/aligner_common.h:147-274). */
typedef struct gzb_engine gzb_engine;

typedef struct {
  int32_t chunk_id;
  int32_t subject_id;   /* sequence index in the chunk */
  int32_t score;        /* reverse + forward gapped score */
  uint32_t hit_q, hit_d;     /* seed: position in query, in chunk */
  uint32_t start_q, start_d; /* alignment start (inclusive) */
  uint32_t end_q, end_d;     /* alignment end (inclusive) */
} gzb_result;

typedef struct {
  uint64_t distance_seeds;     /* representative x check-position pairs */
  uint64_t ungapped_seeds;     /* ungapped extensions run */
  uint64_t ungapped_hits;      /* survivors (score > trigger) */
  uint64_t chained_hits;       /* survivors of the chain filter */
  uint64_t gapped_extensions;  /* one-side extensions */
  uint64_t gapped_cells;       /* DP cells of the gapped extensions */
  uint64_t gapped_fallbacks;   /* extensions the one-thread kernel handed on */
  uint64_t ungapped_steps;     /* residue pairs examined by ungapped X-drop */
  uint64_t kernel_launches;    /* engine kernels launched by the presearch */
} gzb_counters;

/* schedule of the gapped stage (results are identical under every one) */
#define GZB_SCHEDULE_PLAIN 0    /* the static schedule: one launch that deals
                                   the extensions to threads in hit order
                                   (GZB_GAPPED_KERNEL_STATIC), no work queue,
                                   no tile, no model */
#define GZB_SCHEDULE_BATCHED 1  /* persistent kernel of the engine's tile on a
                                   device work queue, extensions ordered
                                   longest-predicted first by the cost model
                                   (hit order when no model is set) */
#define GZB_SCHEDULE_ORACLE 2   /* as BATCHED, ordered by the true costs of
                                   the previous scheduled run of the same
                                   extensions (a measuring stick) */

int gzb_engine_create(int device, gzb_engine **out);
int gzb_engine_destroy(gzb_engine *e);
int gzb_engine_set_params(gzb_engine *e, const gzb_params *p);
/* Uploads one database chunk (concatenated codes with delimiters,
 * offsets[i] = first residue of sequence i, offsets[n] = length) and builds
 * its seed index on the device. */
int gzb_engine_set_database(gzb_engine *e, int32_t chunk_id,
                            const uint8_t *codes, uint64_t length,
                            const uint32_t *offsets,
                            uint32_t number_sequences, void *stream);
/* Device index cache (no counterpart in the reference, which loads the
 * index files its `db` command wrote): gzb_engine_index_bytes gives the
 * size of the resident chunk's index blob, gzb_engine_export_index copies
 * it to host memory, and gzb_engine_set_database_with_index sets a chunk
 * from its codes and such a blob instead of building the index.  The blob
 * records the index parameters and a check of the chunk, and is refused for
 * others. */
int gzb_engine_index_bytes(gzb_engine *e, uint64_t *bytes);
int gzb_engine_export_index(gzb_engine *e, void *blob, uint64_t capacity, void *stream);
int gzb_engine_set_database_with_index(gzb_engine *e, int32_t chunk_id, const uint8_t *codes,
                                       uint64_t length, const uint32_t *offsets,
                                       uint32_t number_sequences, const void *blob,
                                       uint64_t blob_bytes, void *stream);
/* The reference's on-disk seed-searcher index of one chunk (the bytes of
 * its `.sdp` file: SeedSearcherDatabaseParameters::Save,
 * src/seed_searcher_database_parameters.cpp:363-376, written by
 * DatabaseChunk::SaveSeedSearcherParameters, src/database_chunk.h:461-470,
 * and read back by SeedSearcherDatabaseParameters::Build(sequence, length,
 * istream), :321-337) converted to this library's index blob for the chunk
 * (codes / offsets as gzb_engine_set_database), ready for
 * gzb_engine_set_database_with_index.  Host only, no device.  The file must
 * have been built with `params` (clustering, delimiter, window, seed hash,
 * similarity map, cluster threshold) and be consistent; otherwise
 * GZB_ERR_INVALID.  *blob_bytes receives the blob's size; blob = NULL asks
 * only for it. */
int gzb_index_blob_from_reference(const gzb_params *params, const void *sdp, uint64_t sdp_bytes,
                                  const uint8_t *codes, uint64_t length, const uint32_t *offsets,
                                  uint32_t number_sequences, void *blob, uint64_t capacity,
                                  uint64_t *blob_bytes);
/* The seed-index parameters stored in the reference's `.scp` file of a
 * database (SeedSearcherDatabaseParameters::SaveCommonParameters,
 * src/seed_searcher_database_parameters.cpp:378-387) written into *params:
 * delimiter, subsequence_length, map_size, similarity_code_map,
 * hash_code_map, max_indexing_code, code_scores, seed_threshold and
 * max_hash_length.  The other fields are left as the caller set them (the
 * score matrix, gap costs, -b / -v, clustering, min_hash_length and the
 * distance thresholds derived from subsequence_length).  Host only. */
int gzb_params_from_reference_common(const void *scp, uint64_t scp_bytes, gzb_params *params);

/* Stored database chunks, for streaming a database of many chunks
 * (the reference's chunk loop with its preloading thread,
 * src/aligner_gpu_presearch_thread.cpp:214-640 and :259-274, and
 * Database::Preload, src/database.h:556-608).  The engine holds one
 * resident chunk plus up to 64 stored ones, each with its codes, offsets
 * and index arrays.
 *  - gzb_engine_swap_database exchanges the resident chunk with the one in
 *    `slot` (either may be empty): a stored chunk becomes resident without
 *    copies, and the resident one is stored (a chunk whose index was built
 *    here first moves its index arrays out of the build's scratch, one
 *    device copy).  It waits for the work queued on `stream` and for a
 *    prefetch into the slot, and refuses a prefetched chunk with residue
 *    codes of 32 or more.
 *  - gzb_engine_prefetch_database_with_index fills `slot` from host codes,
 *    offsets and an index blob (as gzb_engine_set_database_with_index,
 *    same checks) with asynchronous copies on `stream`, touching only the
 *    slot's own buffers, so the copies overlap a presearch running on
 *    another stream; with pinned host buffers the host does not wait.
 * A database whose chunks all fit in device memory can stay stored
 * (set_database, then swap into its own slot, per chunk); a larger one
 * streams through two slots. */
int gzb_engine_swap_database(gzb_engine *e, uint32_t slot, void *stream);
int gzb_engine_prefetch_database_with_index(gzb_engine *e, uint32_t slot, int32_t chunk_id,
                                            const uint8_t *codes, uint64_t length,
                                            const uint32_t *offsets,
                                            uint32_t number_sequences, const void *blob,
                                            uint64_t blob_bytes, void *stream);

/* Uploads the queries (concatenated, shared delimiters; offsets[i] is the
 * leading delimiter of query i; lengths[i] = residues + 2) with their
 * per-query ungapped X-drop and trigger, and builds the query hash lists. */
int gzb_engine_set_queries(gzb_engine *e, const uint8_t *codes,
                           uint64_t length, const uint32_t *offsets,
                           const uint32_t *lengths, uint32_t number_queries,
                           const int32_t *ungapped_cutoffs,
                           const int32_t *gapped_triggers, void *stream);
/* Query preparation and gzb_engine_set_queries in one call, the prepared
 * codes never leaving the device: protein queries in the engine layout
 * (host codes; with the filter, a letter the reference's SEG does not
 * count, lower case, passed as its code + 32; without it, plain codes below
 * 32) are uploaded, SEG-masked in place when filter is
 * non-zero (gzb_seg_protein_queries; a protein shorter than SEG's window
 * keeps a zero-filled body and the statistics of ProteinQuery's buffer),
 * given their cutoffs by gzb_query_karlin_cutoffs with the engine's score
 * matrix (ungapped_bits / trigger_bits: 7 and 22 for aln), and their hash
 * lists are built.  cutoffs / triggers (optional, host) receive the
 * per-query values.  Replaces Queries::BuildQuery (src/queries.cpp:83-107)
 * and AlignerGpu::SetQueriesData (src/aligner_gpu.cpp:213-242) for -q p.
 * Synchronises `stream`. */
int gzb_engine_set_protein_queries(gzb_engine *e, const uint8_t *codes, uint64_t length,
                                   const uint32_t *offsets, const uint32_t *lengths,
                                   uint32_t number_queries, int filter, float ungapped_bits,
                                   float trigger_bits, int32_t *cutoffs, int32_t *triggers,
                                   void *stream);
/* The same for translated searches (-q d): number_reads reads of ASCII
 * bases, read r = dna[read_offsets[r] .. read_offsets[r + 1]) (host), are
 * uploaded, translated in six frames into the engine's shared-delimiter
 * layout (query r at the offset the reads before it take,
 * gzb_translated_query_length(read length) codes), SEG-masked per frame
 * when filter is non-zero, given their cutoffs and their hash lists.
 * Replaces Queries::BuildQuery with TranslatedDnaQuery
 * (src/translated_dna_query.cpp:44-74) and AlignerGpu::SetQueriesData.
 * Synchronises `stream`. */
int gzb_engine_set_translated_queries(gzb_engine *e, const uint8_t *dna,
                                      const uint64_t *read_offsets, uint32_t number_reads,
                                      int filter, float ungapped_bits, float trigger_bits,
                                      int32_t *cutoffs, int32_t *triggers, void *stream);
/* Runs the presearch of the resident queries against the resident chunk
 * and merges into the per-query top-b lists kept on the device.  Call
 * gzb_engine_reset_results before the first chunk of a query set. */
int gzb_engine_presearch(gzb_engine *e, int schedule, void *stream);
/* Graph mode (no counterpart in the reference, which launches every stage
 * from the host with a round trip per buffer): with graph mode on,
 * gzb_engine_presearch runs the whole presearch of the resident chunk --
 * list lookup, seed search and ungapped extension, hit sort, chain filter,
 * gapped extension, merge -- as one CUDA graph, captured on first use for
 * that chunk, query set, schedule and tile and replayed afterwards (up to
 * 16 graphs per engine, least recently used dropped), with no host
 * synchronisation between stages.  Counts stay on the device and the
 * buffers are sized to capacities for hits and member work (grown by every
 * eager run, or set by gzb_engine_reserve); a run whose counts exceed them
 * merges nothing and is redone eagerly with larger capacities, so results
 * are always those of the eager path.  The cost-model order runs inside
 * the graph (features, prediction and the key sort); the oracle schedule
 * and logging run eagerly.  gzb_engine_get_graph_stats counts captures,
 * graph runs and eager redos. */
int gzb_engine_set_graph(gzb_engine *e, int enable);
int gzb_engine_reserve(gzb_engine *e, uint64_t hits, uint64_t member_work);
int gzb_engine_get_graph_stats(gzb_engine *e, uint64_t *captures, uint64_t *replays,
                               uint64_t *fallbacks);
int gzb_engine_reset_results(gzb_engine *e, void *stream);
/* Copies the merged results to the host: counts[number_queries] and
 * results[number_queries * max_number_results] (row i holds counts[i]
 * valid entries, best first).  Synchronises `stream`. */
int gzb_engine_get_results(gzb_engine *e, uint32_t *counts,
                           gzb_result *results, void *stream);
/* The exchange step of a search whose database chunks are spread over GPUs
 * (one process per GPU, each searching its own chunks): one chunk's lists
 * merged into the running lists on the host, as the reference's
 * AlignerCommon::AddResults (src/aligner_common.h:147-274) merges each
 * chunk's results.  Layout as gzb_engine_get_results.  chunk_counts /
 * chunk_results: one chunk's lists as the engine gives them after
 * gzb_engine_reset_results and one gzb_engine_presearch of that chunk;
 * counts / results: the lists of the chunks merged so far, updated in
 * place.  Merging every chunk this way in chunk order gives exactly the
 * lists of presearching the chunks in turn on one engine.  Host only. */
int gzb_merge_chunk_results(const gzb_params *params, uint32_t number_queries,
                            const uint32_t *chunk_counts, const gzb_result *chunk_results,
                            uint32_t *counts, gzb_result *results);
/* Alignment statistics of one merged result (AlignerCommon::Result,
 * src/aligner_common.h:80-92) as AlignerCommon::BuildResult
 * (src/aligner_common.h:275-340) fills it from the build step's two gapped
 * extensions at the merged result's hit: their summed score, the alignment
 * start and end they reach (concatenated coordinates, end = hit + forward
 * best offset) and what the joined edit path counts.  The build step's
 * X-drop (result_gapped_cutoff) is wider than the presearch's, so score,
 * start and end may exceed the merged result's.  alignment_length == 0
 * marks a result of another chunk (not computed by this call; its score,
 * start and end are then the merged result's). */
typedef struct {
  int32_t chunk_id;
  int32_t subject_id;
  int32_t score;              /* build step: reverse + forward best score */
  uint32_t hit_q, hit_d;      /* the merged result's hit */
  uint32_t start_q, start_d;  /* build step's alignment start */
  uint32_t end_q, end_d;      /* build step's alignment end */
  uint32_t alignment_length;  /* edit ops of the joined path */
  uint32_t mismatches;
  uint32_t gap_openings;
  uint32_t gap_extensions;
  int32_t presearch_score;    /* the merged result's (presearch) score */
} gzb_alignment;
/* The build results step for the resident chunk
 * (AlignerBuildResultsThread::Run, src/aligner_build_results_thread.h:64-190):
 * re-extends both sides of every merged result of this chunk with its edit
 * path (GappedExtender::ExtendOneSide, src/gapped_extender.cpp:70-304, and
 * PickOptimalPath, :473-531) and fills alignments[number_queries *
 * max_number_results] (row i holds counts[i] entries, in result order) on
 * the host.  Synchronises `stream`. */
int gzb_engine_build_alignments(gzb_engine *e, uint32_t *counts, gzb_alignment *alignments,
                                void *stream);
int gzb_engine_get_counters(gzb_engine *e, gzb_counters *out);
/* Device-side ungapped survivors of the last presearch, sorted by
 * (query, database position, query position): copies up to `capacity`
 * triples and returns the total in *count.  Synchronises `stream`. */
int gzb_engine_get_hits(gzb_engine *e, uint32_t *query_ids,
                        uint32_t *query_positions,
                        uint32_t *database_positions, uint64_t capacity,
                        uint64_t *count, void *stream);
/* Device-resident database index arrays (for inspection / tests):
 * which = 0 nc_keys, 1 nc_offsets, 2 nc_values, 3 rep_keys, 4 rep_offsets,
 * 5 rep_cluster_ids, 6 rep_positions, 7 member_offsets,
 * 8 member_positions.  Copies up to `capacity` entries to `out` and returns
 * the element count in *count.  Synchronises `stream`. */
int gzb_engine_get_index_array(gzb_engine *e, int which, uint32_t *out,
                               uint64_t capacity, uint64_t *count,
                               void *stream);
/* Device-resident query hash lists (for inspection / tests): which = 0 list
 * hashes, 1 list offsets (lists + 1), 2 check positions per list (they come
 * first in each list), 3 entry query ids, 4 entry positions within the
 * query.  Same copy semantics as gzb_engine_get_index_array. */
int gzb_engine_get_list_array(gzb_engine *e, int which, uint32_t *out,
                              uint64_t capacity, uint64_t *count, void *stream);
/* Per-extension costs of the last run that used a work-queue schedule
 * (batched, oracle, or plain with logging on), in extension order: the
 * reverse extensions of the chained hits, then the forward ones.  cells:
 * true DP cells (UINT32_MAX for extensions the thread kernel handed to a
 * fallback); predicted: the model's log2(1 + cells), only after a batched
 * run with a model.  *count = extensions; either array may be NULL. */
int gzb_engine_get_extension_costs(gzb_engine *e, float *predicted, uint32_t *cells,
                                   uint64_t capacity, uint64_t *count, void *stream);
/* ---- tile parameters and the autotuner -----------------------------------
 * The first level of the gapped stage runs one extension per thread in one
 * of five kernels (GZB_TILE_GAPPED_KERNEL):
 *   GZB_GAPPED_KERNEL_FLAT  every lane advances one DP cell per step; a lane
 *       at a row or extension boundary waits until GZB_TILE_BOOK_THRESHOLD
 *       lanes of its warp are (or no lane can step), then they do their
 *       bookkeeping together (1..32) and take new extensions from the work
 *       queue, so the lanes of a warp never wait for the slowest extension;
 *   GZB_GAPPED_KERNEL_LANE  each warp takes the next 32 extensions from the
 *       work queue and runs them to completion with a tight row/column loop,
 *       fastest when neighbouring extensions cost the same (the batched
 *       schedule orders them by predicted cost);
 *   GZB_GAPPED_KERNEL_ROWS  each lane runs its extension one database row
 *       per step and takes the next extension from the queue once its own
 *       has ended, so lanes wait for each other only within a row; finished
 *       lanes refill together once GZB_TILE_BOOK_THRESHOLD lanes of the
 *       warp are idle (or none has work left), sharing one round of memory
 *       latency (the process-wide default, threshold 4);
 *   GZB_GAPPED_KERNEL_STATIC  one launch that deals extensions to threads
 *       round-robin, no work queue: the plain schedule's kernel;
 *   GZB_GAPPED_KERNEL_DEAL  the row-step refill of _ROWS with extensions
 *       dealt to lanes round-robin in schedule order instead of queued, so
 *       each lane loads its next extension while it runs the current one;
 *       longest-first order keeps the lanes' totals even.
 * gzb_set_tile_parameter sets the process-wide defaults that the operators
 * and engines without a tuned tile use. */
#define GZB_TILE_BOOK_THRESHOLD 0
#define GZB_TILE_GAPPED_KERNEL 1
/* GZB_TILE_ORDER: the batched schedule's order, GZB_ORDER_MODEL (the cost
 * model's predicted cost, longest first; the default) or GZB_ORDER_HITS
 * (hit order, skipping the features and the prediction). */
#define GZB_TILE_ORDER 2
#define GZB_ORDER_HITS 0
#define GZB_ORDER_MODEL 1
/* GZB_TILE_SEED_WALKER: how the seed search deals its ungapped walks.
 * GZB_SEED_WALKER_UNIT gives each lane whole seed-search units (a
 * representative or residual position with every query position of its
 * list); GZB_SEED_WALKER_DEALT makes the seeds of a warp's 32 units one
 * stream dealt to the lanes 32 at a time, so lanes wait for the longest
 * walk of a round instead of the longest list.  Member seeds are dealt in
 * both.  Results and counters are the same. */
#define GZB_TILE_SEED_WALKER 3
#define GZB_SEED_WALKER_UNIT 0
#define GZB_SEED_WALKER_DEALT 1
/* GZB_TILE_BAND_WIDTH: band columns per lane of the _ROWS kernel, 32, 64
 * (the default) or 128.  The band lives in shared memory (5 bytes per column
 * and lane), so a narrower band fits more blocks on an SM and hands the
 * extensions whose band outgrows it to the warp kernel; a wider one keeps
 * more extensions on one lane with fewer blocks per SM.  Results are the
 * same. */
#define GZB_TILE_BAND_WIDTH 4
#define GZB_GAPPED_KERNEL_FLAT 0
#define GZB_GAPPED_KERNEL_LANE 1
#define GZB_GAPPED_KERNEL_ROWS 2
#define GZB_GAPPED_KERNEL_STATIC 3
#define GZB_GAPPED_KERNEL_DEAL 4
/* GZB_GAPPED_KERNEL_GROUP4 .. _GROUP32: 4, 8, 16 or 32 lanes per extension
 * (the threads-per-extension axis): a group evaluates a database row's band
 * columns that many at a time with shuffle scans (exact for X-drops below
 * 1024, else the _ROWS kernel runs), pulling extensions from the work queue
 * as soon as its own has ended; a band wider than 64 columns goes to the
 * warp kernel. */
#define GZB_GAPPED_KERNEL_GROUP4 5
#define GZB_GAPPED_KERNEL_GROUP8 6
#define GZB_GAPPED_KERNEL_GROUP16 7
#define GZB_GAPPED_KERNEL_GROUP32 8
int gzb_set_tile_parameter(int which, int value);
int gzb_get_tile_parameter(int which, int *value);
/* Per-engine, per-schedule tile: value -1 falls back to the process-wide
 * default.  gzb_engine_autotune stores its pick here. */
int gzb_engine_set_tile(gzb_engine *e, int schedule, int which, int value);
int gzb_engine_get_tile(gzb_engine *e, int schedule, int which, int *value);
/* Times the presearch of the resident queries and chunk under each
 * candidate value (candidates[n]) of tile parameter `which` with
 * `schedule`, keeps the fastest for that schedule (gzb_engine_get_tile) and
 * returns it in *best (ms per candidate in ms[n] if not NULL: the seed
 * search stage's for GZB_TILE_SEED_WALKER, the gapped stage's otherwise).  Runs the presearch twice per candidate and clears the engine's
 * results.  Results are identical under every tile. */
int gzb_engine_autotune(gzb_engine *e, int schedule, int which, const int *candidates,
                        int n, int *best, float *ms, void *stream);

/* ---- cost model of the gapped stage -------------------------------------
 * An 8 -> 32 -> 32 -> 1 ReLU MLP predicts log2(1 + DP cells) of every gapped
 * extension from its ungapped score, ungapped length, positives and
 * identities near the seed, remaining query and subject lengths and
 * direction.  FP32 training with hand-written forward/backward kernels, BF16
 * inference.  Parameters: gzb_cost_model_param_count() floats, layout
 * W1[32][8] b1[32] W2[32][32] b2[32] W3[32] b3. */
int gzb_cost_model_param_count(void);
/* He-normal initial parameters from a seeded generator (host). */
int gzb_cost_model_init(float *params, uint64_t seed);
/* Gradient of the mean squared error over n samples (device buffers:
 * d_x[n][8], d_y[n], d_grad[params]; d_loss receives the mean loss). */
int gzb_cost_model_gradients(const float *d_params, const float *d_x,
                             const float *d_y, uint32_t n, float *d_grad,
                             float *d_loss, void *stream);
/* BF16 inference: d_out[n] predicted log2(1 + cells). */
int gzb_cost_model_predict(const float *d_params, const float *d_x, uint32_t n,
                           float *d_out, void *stream);
/* Minibatch Adam on device-resident samples; params in/out on the host. */
int gzb_cost_model_train(const float *d_x, const float *d_y, uint32_t n,
                         float *params, int epochs, int batch, float lr,
                         uint64_t seed, float *final_loss, void *stream);
/* Logging of (features, log2(1 + cells)) pairs for every gapped extension of
 * the following presearch calls, up to `capacity` pairs (enabling resets
 * the log). */
int gzb_engine_set_logging(gzb_engine *e, int enable, uint64_t capacity);
int gzb_engine_get_log(gzb_engine *e, float *features, float *log_cells,
                       uint64_t capacity, uint64_t *count);
/* Trains a model on the logged pairs (params: host in = initial values,
 * out = trained) and installs it for GZB_SCHEDULE_BATCHED. */
int gzb_engine_train_cost_model(gzb_engine *e, int epochs, int batch, float lr,
                                uint64_t seed, float *params, float *final_loss);
/* Installs host parameters (NULL removes the model). */
int gzb_engine_set_cost_model(gzb_engine *e, const float *params);
/* Mean |predicted - true| log2 cost of the last batched presearch and the
 * number of extensions it covers (-1, 0 when none). */
int gzb_engine_get_schedule_stats(gzb_engine *e, float *mean_abs_log2_error,
                                  uint64_t *count);
/* Time of the last presearch, per stage, in milliseconds (device events):
 * [0] list lookup, [1] seed search + ungapped + sort, [2] chain filter,
 * [3] gapped extension, [4] merge, [5] total, [6] the seed-search kernels
 * alone (part of [1]: seed and member kernels, without the hit sort). */
int gzb_engine_get_stage_ms(gzb_engine *e, float *ms7);


/* ---- query preparation: six-frame translation of DNA reads ----
 * Replaces the per-read TranslatedDnaQuery construction of
 * Queries::BuildQuery (src/queries.cpp:83-107; layout
 * src/translated_dna_query.cpp:44-74, codons src/translator.cpp:104-142)
 * with filtering off.  gzb_translated_query_length gives a read's
 * translated query length in codes, both delimiters included
 * (TranslatedDnaQuery::GetSequenceLength, src/translated_dna_query.h:24-31;
 * a read shorter than 3 bases gives 2, an empty query, where the reference
 * writes past an empty buffer).  gzb_translate_dna_queries translates
 * number_reads reads held on the device (ASCII, read r = d_dna[d_offsets[r]
 * .. + d_lengths[r])) into d_out, query r starting at d_out_offsets[r]; to
 * get the engine's shared-delimiter layout set d_out_offsets[r + 1] =
 * d_out_offsets[r] + gzb_translated_query_length(length r) - 1.  Reads
 * nothing back; asynchronous on `stream`. */
uint64_t gzb_translated_query_length(uint32_t length);
int gzb_translate_dna_queries(const uint8_t *d_dna, const uint64_t *d_offsets,
                              const uint32_t *d_lengths, uint32_t number_reads,
                              const uint64_t *d_out_offsets, uint8_t delimiter,
                              uint8_t *d_out, void *stream);


/* ---- query preparation: per-query Karlin-Altschul cutoffs ----
 * Replaces the per-query SetStaticalParameters of ProteinQuery and
 * TranslatedDnaQuery (Statistics::CalculateUngappedKarlinParameters,
 * src/statistics.cpp:205-229, over ext/karlin/src/karlin.c) and the cutoff
 * conversion of AlignerGpu::SetQueriesData (src/aligner_gpu.cpp:228-238):
 * for query r (codes d_codes[d_offsets[r] .. + d_lengths[r]), delimiters
 * included) it computes lambda, K and H of its composition against the
 * Robinson background and writes
 *   d_cutoffs[r]  = floor(ungapped_bits * ln2 / lambda)           (X-drop)
 *   d_triggers[r] = floor((trigger_bits * ln2 + ln K) / lambda)   (trigger)
 * and, when d_karlin is not NULL, d_karlin[3r..3r+2] = lambda, K, H.  The
 * aln defaults are ungapped_bits 7 and trigger_bits 22.  score_matrix is
 * the host number_letters^2 protein matrix (20 regular letters first; at
 * most 32 letters and a score range of at most 31).  Asynchronous on
 * `stream`; nothing is allocated. */
int gzb_query_karlin_cutoffs(const uint8_t *d_codes, const uint64_t *d_offsets,
                             const uint32_t *d_lengths, uint32_t number_queries,
                             const int32_t *score_matrix, uint32_t number_letters,
                             float ungapped_bits, float trigger_bits, int32_t *d_cutoffs,
                             int32_t *d_triggers, float *d_karlin, void *stream);


/* ---- query preparation: SEG low-complexity masking (aln -F T, the
 * default) ----
 * Replaces SequenceSegFilter (src/sequence_seg_filter.cpp:17-23 over
 * ext/seg/src/seg.cpp, window 12) as the query builders apply it, in place
 * on device query codes:
 *  - gzb_seg_translated_queries masks the six frames of each translated
 *    query written by gzb_translate_dna_queries (d_query_offsets = its
 *    d_out_offsets, d_read_lengths = the reads' base counts); a frame of
 *    fewer than 12 codons becomes unknown codes
 *    (src/translated_dna_query.cpp:56-73);
 *  - gzb_seg_protein_queries masks the body of each protein query in the
 *    engine layout (d_offsets = leading delimiter, d_lengths = residues +
 *    2); a protein of fewer than 12 residues gets a body of code 0, the
 *    zero-filled buffer ProteinQuery keeps when the filter refuses it
 *    (src/protein_query.cpp:39-49).  Only codes 0-19 count as amino acids;
 *    a caller that must keep a letter out of the compositions (the
 *    reference's SEG ignores lower-case letters) passes its code + 32,
 *    which comes back as the code.
 * Masked residues become the unknown code 24.  d_status (optional, one
 * zeroed uint32 on the device) counts sequences left unmasked because they
 * exceed 65535 residues or nest the search deeper than the kernel's stack.
 * The first call on a device uploads a 512 KB table (synchronously); later
 * calls are asynchronous on `stream`. */
int gzb_seg_translated_queries(uint8_t *d_queries, const uint64_t *d_query_offsets,
                               const uint32_t *d_read_lengths, uint32_t number_queries,
                               uint32_t *d_status, void *stream);
int gzb_seg_protein_queries(uint8_t *d_codes, const uint64_t *d_offsets,
                            const uint32_t *d_lengths, uint32_t number_queries,
                            uint32_t *d_status, void *stream);


/* ---- the final hit table (host functions, no device) ----
 * What AlignerCommon::WriteOutput (src/aligner_common.h:344-394) prints
 * beside a result's alignment statistics:
 *  - gzb_gapped_karlin_parameters: lambda, K, H and the length-adjustment
 *    alpha, beta of the gapped protein search
 *    (Statistics::CalculateGappedKarlinParameters / CalculateAlphaBeta,
 *    src/statistics.cpp:232-270; BLOSUM62 11/1 and PAM30 9/1);
 *  - gzb_search_space: a query's search space with the length adjustment
 *    (Statistics::CalculateSearchSpace, src/statistics.cpp:50-122);
 *    query_length is the query's real length (residues; a read's bases / 3
 *    for a translated query), db_length and db_sequences those of the whole
 *    database (residues without delimiters, all chunks);
 *  - gzb_evalue / gzb_bit_score: Statistics::Nominal2EValue and
 *    Nominal2Normalized (src/statistics.cpp:23-48);
 *  - gzb_translated_real_start / _end: a translated query position's base
 *    in the read (TranslatedDnaQuery::GetRealStart / GetRealEnd,
 *    src/translated_dna_query.h:43-61); protein query positions are their
 *    own real positions. */
int gzb_gapped_karlin_parameters(const char *matrix_name, int gap_open, int gap_extension,
                                 float *lambda, float *k, float *h, double *alpha,
                                 double *beta);
uint64_t gzb_search_space(uint64_t query_length, uint64_t db_length, uint64_t db_sequences,
                          float lambda, float k, double alpha, double beta);
double gzb_evalue(int32_t score, uint64_t search_space, float lambda, float k);
float gzb_bit_score(int32_t score, float lambda, float k);
uint32_t gzb_translated_real_start(uint32_t position, uint32_t dna_length);
uint32_t gzb_translated_real_end(uint32_t position, uint32_t dna_length);
/* The tabular lines AlignerCommon::WriteOutput (src/aligner_common.h:344-394)
 * prints for the alignment records of gzb_engine_build_alignments (counts,
 * rows of `stride` records per query; rows with alignment_length 0 are
 * skipped), one '\n'-terminated line per result: query name, subject name,
 * identity %, alignment length, mismatches, gap openings, query start and
 * end (read bases when dna_lengths is given), subject start and end,
 * E-value, normalized score.  db_offsets: the chunk's first-residue offsets
 * (subject_id indexes them and subject_names); db_length / db_sequences:
 * residues and sequences of the whole database; query_real_lengths as for
 * gzb_search_space; lambda, k, alpha, beta from
 * gzb_gapped_karlin_parameters.  *written receives the bytes of the text;
 * out = NULL asks only for it.  Host only. */
/* The last step of the build results stage before the table is written
 * (AlignerBuildResultsThread::Run, src/aligner_build_results_thread.h:179-190):
 * each query's alignment records reordered in place by
 * AlignerCommon::ResultGreaterScore (src/aligner_common.h:116-121,
 * src/aligner_common.cpp:12-52): higher score first, then the longer
 * query span, the longer subject span, the smaller subject-relative start;
 * spans are the uint32 differences of the printed coordinates (read bases
 * for translated queries).  The records must be in merged-result order
 * (the order of gzb_engine_get_results), which is the order the reference
 * sorts from; the sort is std::sort with that comparator, as the
 * reference's.  Arguments as for gzb_write_hit_table.  Host only. */
int gzb_sort_alignments(uint32_t number_queries, uint32_t stride, const uint32_t *counts,
                        gzb_alignment *alignments, uint32_t number_subjects,
                        const uint32_t *db_offsets, const uint32_t *dna_lengths);
int gzb_write_hit_table(uint32_t number_queries, uint32_t stride, const uint32_t *counts,
                        const gzb_alignment *alignments, const char *const *query_names,
                        const char *const *subject_names, uint32_t number_subjects,
                        const uint32_t *db_offsets, uint64_t db_length, uint64_t db_sequences,
                        const uint32_t *query_real_lengths, const uint32_t *dna_lengths,
                        float lambda, float k, double alpha, double beta, char *out,
                        uint64_t capacity, uint64_t *written);

#ifdef __cplusplus
}
#endif
#endif
