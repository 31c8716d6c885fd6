/*
 * gz_oracle.c -- CPU restatement of the GHOSTZ-GPU presearch path.
 *
 * TEST INFRASTRUCTURE ONLY (see gz_oracle.h).  Sequential C; each function
 * cites the reference file:line whose behaviour it restates.  Paths are
 * relative to the reference project root.
 */
#include "gz_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define GZO_INIT_SCORE (-(1 << 10)) /* src/gapped_extender.h:40 */

static void *xmalloc(size_t n) {
  void *p = malloc(n ? n : 1);
  if (!p) abort();
  return p;
}
static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s ? s : 1);
  if (!p) abort();
  return p;
}

/* ------------------------------------------------------------------ */
/* Variable-length reduced-alphabet hash.
 * Restates ReducedAlphabetVariableHashFunction::CalculateHash
 * (src/reduced_alphabet_variable_hash_function.cpp:56-86) together with the
 * constructor's code+1 shift and shift-size rule (:18-43, :109-115).
 * A residue is hashable when its reduced code is <= max_indexing_code; the
 * validity test of residue k comes before the length/score stop test, so a
 * k-mer whose next residue is unhashable fails even when already complete. */
static uint32_t hash_shift(const gzo_params *p) {
  uint32_t max_code = (uint32_t)p->max_indexing_code + 1u;
  uint32_t shift = 0;
  for (uint32_t c = 1; c < max_code; c <<= 1) ++shift;
  return shift;
}

int gzo_hash(const gzo_params *p, const uint8_t *seq, uint32_t *hash,
             uint32_t *hash_length) {
  const uint32_t shift = hash_shift(p);
  uint32_t h = 0;
  int score = 0;
  int32_t k;
  for (k = 0; k < p->max_hash_length; ++k) {
    uint8_t c = seq[k];
    if (c >= p->map_size || p->hash_code_map[c] > p->max_indexing_code) {
      *hash = 0;
      *hash_length = 0;
      return 1;
    }
    if (k >= p->min_hash_length && score >= p->seed_threshold) break;
    uint32_t r = (uint32_t)p->hash_code_map[c] + 1u;
    h = (h << shift) + r;
    score += p->code_scores[r - 1u];
  }
  *hash = h;
  *hash_length = (uint32_t)k;
  return 0;
}

/* ------------------------------------------------------------------ */
/* Reduced-alphabet Hamming distance over an L window centred on the seed.
 * Restates DistanceCalculator::CalculateDistance
 * (src/distance_calculator.cpp:35-54): window = center - L/2 ... +L. */
int gzo_distance(const gzo_params *p, const uint8_t *seq0, uint32_t center0,
                 const uint8_t *seq1, uint32_t center1) {
  const uint32_t L = (uint32_t)p->subsequence_length;
  const uint8_t *a = seq0 + center0 - L / 2;
  const uint8_t *b = seq1 + center1 - L / 2;
  int mismatches = 0;
  for (uint32_t i = 0; i < L; ++i)
    mismatches += p->similarity_code_map[a[i]] != p->similarity_code_map[b[i]];
  return mismatches;
}

/* ------------------------------------------------------------------ */
/* Ungapped one-side X-drop, score only.
 * Restates UngappedExtender::ExtendOneSideScoreOnly
 * (src/ungapped_extender.h:34-82): the best score is the best prefix sum;
 * the walk stops at a delimiter on either side or once the running sum
 * since the last best drops to -cutoff or below. */
int gzo_ungapped_one_side(const gzo_params *p, const uint8_t *seq0,
                          const uint8_t *seq1, int reversed, int cutoff) {
  const int inc = reversed ? -1 : 1;
  const int delim = p->delimiter;
  const int n = p->number_letters;
  const int32_t *sm = p->score_matrix;
  int pos = 0;
  int best = 0;
  if (seq1[0] == delim || seq0[0] == delim) return 0;
  int run = 0; /* sum since the last improvement */
  for (;;) {
    if (seq1[pos] == delim || seq0[pos] == delim) break;
    run += sm[seq1[pos] * n + seq0[pos]];
    pos += inc;
    if (run > 0) {
      best += run;
      run = 0;
      /* the reference keeps adding single positive steps directly */
      for (;;) {
        if (seq1[pos] == delim || seq0[pos] == delim) {
          run = 0;
          goto done;
        }
        int s = sm[seq1[pos] * n + seq0[pos]];
        pos += inc;
        if (s > 0) {
          best += s;
        } else {
          run = s;
          break;
        }
      }
    }
    if (!(run > -cutoff)) break;
  }
done:
  return best;
}

/* Reverse extension from (q-1, d-1); forward from (q, d) only when the
 * reverse score has not yet passed the trigger.  Restates
 * SeedSearcher::UngappedExtend (src/seed_searcher.h:133-158). */
int gzo_ungapped_with_trigger(const gzo_params *p, const uint8_t *query,
                              uint32_t query_position, const uint8_t *db,
                              uint32_t db_position, int cutoff, int trigger) {
  int sum = gzo_ungapped_one_side(p, query + query_position - 1,
                                  db + db_position - 1, 1, cutoff);
  if (sum <= trigger)
    sum += gzo_ungapped_one_side(p, query + query_position,
                                 db + db_position, 0, cutoff);
  return sum;
}

/* ------------------------------------------------------------------ */
/* Affine-gap X-drop extension, score only.
 * Restates GappedExtender::ExtendOneSideScoreOnly
 * (src/gapped_extender.cpp:306-471).  Rows follow seq1 (database), columns
 * follow seq0 (query); column c holds query residue (c-1)*inc.  best/gap
 * arrays are the reference's DpCell{best, best_gap}.  The band is
 * [array_start, array_end); cells are pruned against the running maximum
 * as each cell is evaluated, in row order. */
int gzo_gapped_one_side(const gzo_params *p, const uint8_t *seq0,
                        const uint8_t *seq1, int reversed, int cutoff,
                        int *best_score, int *best_pos0, int *best_pos1,
                        uint64_t *cells) {
  const int inc = reversed ? -1 : 1;
  const int delim = p->delimiter;
  const int n = p->number_letters;
  const int gap_ext = p->gap_extension;
  const int gap_init = p->gap_open + p->gap_extension;
  uint64_t cell_count = 0;

  *best_score = 0;
  *best_pos0 = -inc;
  *best_pos1 = -inc;
  if (cells) *cells = 0;
  if (seq0[0] == delim || seq1[0] == delim) return 0;

  /* column count: residues of seq0 up to its delimiter, plus col 0 and one
   * sentinel */
  int len0 = 0;
  while (seq0[len0 * inc] != delim) ++len0;
  int *best = (int *)xmalloc(sizeof(int) * (size_t)(len0 + 2));
  int *gap = (int *)xmalloc(sizeof(int) * (size_t)(len0 + 2));

  /* row -1: the leading horizontal gap run, cut at -cutoff (:345-364) */
  int score = -gap_init;
  int col = 1;
  int pos0 = 0;
  best[0] = 0;
  gap[0] = -gap_init;
  for (; seq0[pos0] != delim; ++col, pos0 += inc) {
    if (score < -cutoff) break;
    best[col] = score;
    gap[col] = score - gap_init;
    score -= gap_ext;
  }
  int band_start = 0, band_end;
  if (seq0[pos0] != delim) {
    best[col] = GZO_INIT_SCORE;
    gap[col] = GZO_INIT_SCORE;
    band_end = col + 1;
  } else {
    band_end = col;
  }

  int max_score = 0;
  int max_pos0 = -inc, max_pos1 = -inc;
  int pos1;
  for (pos1 = 0; seq1[pos1] != delim; pos1 += inc) {
    const int32_t *mrow = p->score_matrix + seq1[pos1] * n;
    int last_kept;
    int row_gap; /* horizontal gap entering the next cell */
    int diag;
    pos0 = band_start * inc;
    diag = best[band_start];
    /* column band_start only receives the vertical gap (:400-407) */
    if (max_score - gap[band_start] > cutoff)
      best[band_start] = GZO_INIT_SCORE;
    else
      best[band_start] = gap[band_start];
    row_gap = best[band_start] - gap_init;
    gap[band_start] -= gap_ext;
    last_kept = band_start;
    for (col = band_start + 1; col < band_end; ++col, pos0 += inc) {
      int s = diag + mrow[seq0[pos0]];
      int vgap = gap[col];
      diag = best[col];
      ++cell_count;
      if (s < vgap) s = vgap;
      if (s < row_gap) s = row_gap;
      if (max_score - s > cutoff) {
        if (band_start + 1 == col) ++band_start;
        best[col] = GZO_INIT_SCORE;
        gap[col] = GZO_INIT_SCORE;
        row_gap = GZO_INIT_SCORE;
      } else {
        last_kept = col;
        if (s > max_score) {
          max_score = s;
          max_pos0 = pos0;
          max_pos1 = pos1;
        }
        gap[col] = (s - gap_init > vgap - gap_ext) ? s - gap_init
                                                   : vgap - gap_ext;
        row_gap = (s - gap_init > row_gap - gap_ext) ? s - gap_init
                                                     : row_gap - gap_ext;
        best[col] = s;
      }
    }
    if (band_start + 1 == band_end) break; /* (:445-447) */
    if (last_kept < band_end - 1) {
      /* shrink the right edge; pos0 still names the old edge (:449-450) */
      band_end = last_kept + 1;
    } else {
      /* grow the right edge along the horizontal gap (:452-459) */
      while (row_gap >= max_score - cutoff && seq0[pos0] != delim) {
        best[band_end] = row_gap;
        gap[band_end] = row_gap - gap_init;
        row_gap -= gap_ext;
        ++band_end;
        pos0 += inc;
        ++cell_count;
      }
    }
    if (seq0[pos0] != delim) { /* sentinel column (:461-465) */
      best[band_end] = GZO_INIT_SCORE;
      gap[band_end] = GZO_INIT_SCORE;
      ++band_end;
    }
  }
  free(best);
  free(gap);
  *best_score = max_score;
  *best_pos0 = max_pos0;
  *best_pos1 = max_pos1;
  if (cells) *cells = cell_count;
  return 0;
}

/* ------------------------------------------------------------------ */

/* Edit ops of the DP (src/gapped_extender.h:46-52) */
enum { TB_SUB = 0, TB_GAP0 = 1, TB_GAP1 = 2, TB_EXT0 = 4, TB_EXT1 = 8 };

/* GappedExtender::ExtendOneSide with an edit script
 * (src/gapped_extender.cpp:70-304): the score-only recurrence plus one op
 * byte per kept cell, stored per row for the band's columns; then
 * PickOptimalPath (:473-531) from the best cell back to the origin. */
int gzo_gapped_one_side_edits(const gzo_params *p, const uint8_t *seq0,
                              const uint8_t *seq1, int reversed, int cutoff,
                              int *best_score, int *best_pos0, int *best_pos1,
                              uint8_t *ops, size_t ops_cap, size_t *n_ops) {
  const int inc = reversed ? -1 : 1;
  const int delim = p->delimiter;
  const int n = p->number_letters;
  const int gap_ext = p->gap_extension;
  const int gap_init = p->gap_open + p->gap_extension;
  *best_score = 0;
  *best_pos0 = -inc;
  *best_pos1 = -inc;
  *n_ops = 0;
  if (seq0[0] == delim || seq1[0] == delim) return 0;
  int len0 = 0, len1 = 0;
  while (seq0[len0 * inc] != delim) ++len0;
  while (seq1[len1 * inc] != delim) ++len1;
  int *best = (int *)xmalloc(sizeof(int) * (size_t)(len0 + 2));
  int *gap = (int *)xmalloc(sizeof(int) * (size_t)(len0 + 2));
  /* per row r: ops of columns [row_start[r], row_start[r] + row_len[r]) at
   * arena + row_off[r]; op bytes of pruned cells stay unset (never read) */
  size_t arena_cap = 1024, arena_used = 0;
  uint8_t *arena = (uint8_t *)calloc(arena_cap, 1);
  if (!arena) abort();
  size_t *row_off = (size_t *)xmalloc(sizeof(size_t) * (size_t)(len1 + 1));
  int *row_start = (int *)xmalloc(sizeof(int) * (size_t)(len1 + 1));
  int score = -gap_init, col = 1, pos0 = 0;
  best[0] = 0;
  gap[0] = -gap_init;
  for (; seq0[pos0] != delim; ++col, pos0 += inc) {
    if (score < -cutoff) break;
    best[col] = score;
    gap[col] = score - gap_init;
    score -= gap_ext;
  }
  int band_start = 0, band_end;
  if (seq0[pos0] != delim) {
    best[col] = GZO_INIT_SCORE;
    gap[col] = GZO_INIT_SCORE;
    band_end = col + 1;
  } else {
    band_end = col;
  }
  int max_score = 0, max_pos0 = -inc, max_pos1 = -inc;
  int pos1, r = 0;
  for (pos1 = 0; seq1[pos1] != delim; pos1 += inc, ++r) {
    /* room for this row: the band can grow by at most the remaining seq0 */
    const size_t need = (size_t)(len0 + 2 - band_start);
    while (arena_used + need > arena_cap) {
      arena = (uint8_t *)realloc(arena, arena_cap * 2);
      if (!arena) abort();
      memset(arena + arena_cap, 0, arena_cap);
      arena_cap *= 2;
    }
    row_off[r] = arena_used;
    row_start[r] = band_start;
    uint8_t *row_ops = arena + arena_used - band_start; /* indexed by column */
    const int32_t *mrow = p->score_matrix + seq1[pos1] * n;
    pos0 = band_start * inc;
    int diag = best[band_start];
    if (max_score - gap[band_start] > cutoff)
      best[band_start] = GZO_INIT_SCORE;
    else
      best[band_start] = gap[band_start];
    int row_gap = best[band_start] - gap_init;
    gap[band_start] -= gap_ext;
    row_ops[band_start] = TB_GAP0 + TB_EXT0;
    int last_kept = band_start;
    for (col = band_start + 1; col < band_end; ++col, pos0 += inc) {
      int s = diag + mrow[seq0[pos0]];
      const int vgap = gap[col];
      diag = best[col];
      int op = TB_SUB;
      if (s < vgap) { op = TB_GAP0; s = vgap; }
      if (s < row_gap) { op = TB_GAP1; s = row_gap; }
      if (max_score - s > cutoff) {
        if (band_start + 1 == col) ++band_start;
        best[col] = GZO_INIT_SCORE;
        gap[col] = GZO_INIT_SCORE;
        row_gap = GZO_INIT_SCORE;
      } else {
        last_kept = col;
        if (s > max_score) {
          max_score = s;
          max_pos0 = pos0;
          max_pos1 = pos1;
        }
        /* a tie between opening and extending counts as extending (:426-437) */
        if (vgap - gap_ext < s - gap_init) {
          gap[col] = s - gap_init;
        } else {
          gap[col] = vgap - gap_ext;
          op += TB_EXT0;
        }
        if (row_gap - gap_ext < s - gap_init) {
          row_gap = s - gap_init;
        } else {
          row_gap -= gap_ext;
          op += TB_EXT1;
        }
        row_ops[col] = (uint8_t)op;
        best[col] = s;
      }
    }
    if (band_start + 1 == band_end) { ++r; break; }
    if (last_kept < band_end - 1) {
      band_end = last_kept + 1;
    } else {
      while (row_gap >= max_score - cutoff && seq0[pos0] != delim) {
        best[band_end] = row_gap;
        gap[band_end] = row_gap - gap_init;
        row_ops[band_end] = TB_GAP0 + TB_EXT0;
        row_gap -= gap_ext;
        ++band_end;
        pos0 += inc;
      }
    }
    if (seq0[pos0] != delim) {
      best[band_end] = GZO_INIT_SCORE;
      gap[band_end] = GZO_INIT_SCORE;
      ++band_end;
    }
    /* the row keeps (final band end - its start) bytes, sentinel slot
     * included, as the reference's gap-state accounting does (:464-466) */
    arena_used += (size_t)(band_end - row_start[r]);
  }
  *best_score = max_score;
  *best_pos0 = max_pos0;
  *best_pos1 = max_pos1;
  /* PickOptimalPath: positions in units of inc (row = pos1 * inc, c0 = pos0 * inc) */
  size_t m = 0;
  int ok = 1;
#define TB_PUSH(o)                          \
  do {                                      \
    if (m >= ops_cap) { ok = 0; goto tb_done; } \
    ops[m++] = (uint8_t)(o);                \
  } while (0)
  {
    int op = TB_SUB;
    int rr = max_pos1 * inc, c0 = max_pos0 * inc;
    while (rr >= 0 && c0 >= 0) {
      const int next = arena[row_off[rr] + (size_t)(c0 + 1 - row_start[rr])];
      if (op == TB_GAP0) {
        op = next & 3;
        if (next & TB_EXT0) op = TB_GAP0;
      } else if (op == TB_GAP1) {
        op = next & 3;
        if (next & TB_EXT1) op = TB_GAP1;
      } else {
        op = next & 3;
      }
      if (op == TB_GAP0) {
        TB_PUSH(GZO_OP_GAP0);
        --rr;
      } else if (op == TB_GAP1) {
        TB_PUSH(GZO_OP_GAP1);
        --c0;
      } else {
        TB_PUSH(GZO_OP_SUB);
        --rr;
        --c0;
      }
    }
    for (; rr >= 0; --rr) TB_PUSH(GZO_OP_GAP0);
    for (; c0 >= 0; --c0) TB_PUSH(GZO_OP_GAP1);
  }
tb_done:
#undef TB_PUSH
  /* the path was collected from the best cell back to the origin; a forward
   * side is reversed to run from the origin (EditBlocks::Reverse) */
  if (ok && inc > 0)
    for (size_t i = 0, j = m ? m - 1 : 0; i < j; ++i, --j) {
      const uint8_t t = ops[i];
      ops[i] = ops[j];
      ops[j] = t;
    }
  *n_ops = m;
  free(best);
  free(gap);
  free(arena);
  free(row_off);
  free(row_start);
  return ok ? 0 : -1;
}

/* AlignerBuildResultsThread::Run (src/aligner_build_results_thread.h:110-160)
 * and AlignerCommon::BuildResult (src/aligner_common.h:275-340). */
int gzo_build_alignment(const gzo_params *p, const uint8_t *query, uint32_t hit_q,
                        const uint8_t *db, uint32_t hit_d, gzo_alignment *out) {
  size_t cap = 1 << 16;
  uint8_t *rev = (uint8_t *)xmalloc(cap), *fwd = (uint8_t *)xmalloc(cap);
  size_t nr = 0, nf = 0;
  int sr, r0, r1, sf, f0, f1;
  /* the build results step's X-drop is normalized_result_gapped_extension_cutoff
   * (src/aligner_gpu.cpp:254-256, src/aligner.cpp), not the presearch one */
  const int cutoff = p->result_gapped_cutoff;
  int rc = gzo_gapped_one_side_edits(p, query + hit_q - 1, db + hit_d - 1, 1, cutoff,
                                     &sr, &r0, &r1, rev, cap, &nr);
  if (rc == 0)
    rc = gzo_gapped_one_side_edits(p, query + hit_q, db + hit_d, 0, cutoff, &sf, &f0,
                                   &f1, fwd, cap, &nf);
  if (rc != 0) {
    free(rev);
    free(fwd);
    return -1;
  }
  out->score = sr + sf;
  out->start_q = hit_q - 1 + (uint32_t)r0;
  out->start_d = hit_d - 1 + (uint32_t)r1;
  out->end_q = hit_q + (uint32_t)f0;
  out->end_d = hit_d + (uint32_t)f1;
  /* the reverse side's path runs from the hit toward the start: reversed,
   * it starts at `start`; the forward path follows */
  uint32_t qp = out->start_q, dp = out->start_d, mm = 0, o = 0, e = 0;
  int prev = GZO_OP_SUB;
  for (size_t i = 0; i < nr + nf; ++i) {
    const int op = i < nr ? rev[nr - 1 - i] : fwd[i - nr];
    if (op == GZO_OP_SUB) {
      if (query[qp] != db[dp]) ++mm;
      ++qp;
      ++dp;
    } else if (op == GZO_OP_GAP0) {
      if (prev != GZO_OP_GAP0) ++o; else ++e;
      ++dp;
    } else {
      if (prev != GZO_OP_GAP1) ++o; else ++e;
      ++qp;
    }
    prev = op;
  }
  out->alignment_length = (uint32_t)(nr + nf);
  out->mismatches = mm;
  out->gap_openings = o;
  out->gap_extensions = e;
  free(rev);
  free(fwd);
  return 0;
}

/* Chain filter.  Restates ChainFilter::Filter / Connected
 * (src/chain_filter.cpp:24-99).  Hits are ordered by database position;
 * the reference's std::sort leaves equal database positions in an
 * unspecified order, and such hits always fall on different diagonal slots,
 * so the kept set does not depend on it.  This restatement breaks the tie by
 * query position to fix the output order. */
typedef struct {
  uint32_t q, d;
} hit_qd;

static int cmp_hit_dq(const void *a, const void *b) {
  const hit_qd *x = (const hit_qd *)a, *y = (const hit_qd *)b;
  if (x->d != y->d) return x->d < y->d ? -1 : 1;
  if (x->q != y->q) return x->q < y->q ? -1 : 1;
  return 0;
}

static int chain_connected(const gzo_params *p, const uint8_t *query,
                           const uint8_t *db, uint32_t chain_query_end,
                           uint32_t hq, uint32_t hd, int cutoff) {
  if (hq <= chain_query_end + 1) return 1;
  const int delim = p->delimiter;
  const int n = p->number_letters;
  uint32_t qo = hq, dof = hd;
  int score = 0, best = 0, c = -cutoff;
  do {
    --dof;
    --qo;
    if (db[dof] == delim || query[qo] == delim || qo <= chain_query_end) break;
    score += p->score_matrix[db[dof] * n + query[qo]];
    if (best < score) {
      best = score;
      c = best - cutoff;
    }
  } while (score > c);
  return qo <= chain_query_end;
}

size_t gzo_chain_filter(const gzo_params *p, const uint8_t *query,
                        uint32_t query_length, int cutoff, const uint8_t *db,
                        uint32_t *hit_q, uint32_t *hit_d, size_t n) {
  hit_qd *h = (hit_qd *)xmalloc(sizeof(hit_qd) * n);
  for (size_t i = 0; i < n; ++i) {
    h[i].q = hit_q[i];
    h[i].d = hit_d[i];
  }
  qsort(h, n, sizeof(hit_qd), cmp_hit_dq);
  uint32_t *slot_diag = (uint32_t *)xcalloc(query_length, sizeof(uint32_t));
  uint32_t *slot_end = (uint32_t *)xcalloc(query_length, sizeof(uint32_t));
  size_t kept = 0;
  for (size_t i = 0; i < n; ++i) {
    uint32_t diagonal = query_length - 1 + h[i].d - h[i].q;
    uint32_t slot = diagonal % query_length;
    if (slot_diag[slot] != diagonal ||
        !chain_connected(p, query, db, slot_end[slot], h[i].q, h[i].d,
                         cutoff)) {
      slot_end[slot] = h[i].q;
      slot_diag[slot] = diagonal;
      hit_q[kept] = h[i].q;
      hit_d[kept] = h[i].d;
      ++kept;
    } else {
      slot_end[slot] = h[i].q;
    }
  }
  free(slot_diag);
  free(slot_end);
  free(h);
  return kept;
}

/* ------------------------------------------------------------------ */
/* Database index with subsequence clustering.
 * Restates SeedSearcherDatabaseParameters::Build
 * (src/seed_searcher_database_parameters.cpp:41-319) and the inverted
 * indexes it fills (src/dense_hash_inverted_index.h:101-135,
 * src/perfect_hash_inverted_index.h:60-84).  Keys are kept sorted here
 * (the reference keeps them in a hash map), values per key stay in
 * database-position order as in the reference, and cluster ids are
 * numbered in (hash, position) order; the reference numbers them in hash
 * map iteration order, which changes no seed. */
struct gzo_db_index {
  uint32_t *arr[9];
  size_t len[9];
};

enum { ST_UNSET = 0, ST_NON_CLUSTERING = 1, ST_REP = 2, ST_MEMBER = 3 };

static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* Build key/offset/value CSR from (hash<<32|value) pairs sorted ascending. */
static void csr_from_pairs(const uint64_t *pairs, size_t n, uint32_t **keys,
                           size_t *nkeys, uint32_t **offsets,
                           uint32_t **values) {
  size_t k = 0;
  for (size_t i = 0; i < n; ++i)
    if (i == 0 || (pairs[i] >> 32) != (pairs[i - 1] >> 32)) ++k;
  *keys = (uint32_t *)xmalloc(sizeof(uint32_t) * k);
  *offsets = (uint32_t *)xmalloc(sizeof(uint32_t) * (k + 1));
  *values = (uint32_t *)xmalloc(sizeof(uint32_t) * n);
  k = 0;
  for (size_t i = 0; i < n; ++i) {
    if (i == 0 || (pairs[i] >> 32) != (pairs[i - 1] >> 32)) {
      (*keys)[k] = (uint32_t)(pairs[i] >> 32);
      (*offsets)[k] = (uint32_t)i;
      ++k;
    }
    (*values)[i] = (uint32_t)pairs[i];
  }
  (*offsets)[k] = (uint32_t)n;
  *nkeys = k;
}

gzo_db_index *gzo_db_index_build(const gzo_params *p, const uint8_t *db,
                                 uint32_t length) {
  gzo_db_index *x = (gzo_db_index *)xcalloc(1, sizeof(gzo_db_index));
  /* 1. hash every position; drop a k-mer that the next one is contained in
   *    (:85-108: the later, contained k-mer replaces the earlier one). */
  uint64_t *pairs = (uint64_t *)xmalloc(sizeof(uint64_t) * (size_t)length);
  size_t np = 0;
  uint32_t prev_len = 0;
  for (uint32_t i = 0; i < length; ++i) {
    uint32_t h, hl;
    if (!gzo_hash(p, db + i, &h, &hl)) {
      uint64_t pr = ((uint64_t)h << 32) | i;
      if (prev_len != 0 && prev_len - 1 >= hl)
        pairs[np - 1] = pr;
      else
        pairs[np++] = pr;
      prev_len = hl;
    } else {
      prev_len = 0;
    }
  }
  qsort(pairs, np, sizeof(uint64_t), cmp_u64);

  if (!p->clustering) {
    csr_from_pairs(pairs, np, &x->arr[0], &x->len[0], &x->arr[1], &x->arr[2]);
    x->len[1] = x->len[0] + 1;
    x->len[2] = np;
    x->arr[3] = (uint32_t *)xmalloc(4);
    x->arr[4] = (uint32_t *)xcalloc(1, 4);
    x->len[4] = 1;
    x->arr[5] = (uint32_t *)xmalloc(4);
    x->arr[6] = (uint32_t *)xmalloc(4);
    x->arr[7] = (uint32_t *)xcalloc(1, 4);
    x->len[7] = 1;
    x->arr[8] = (uint32_t *)xmalloc(4);
    free(pairs);
    return x;
  }

  /* 2. clustering within each hash bucket (:109-205) */
  const uint32_t L = (uint32_t)p->subsequence_length;
  const uint32_t half = L / 2;
  uint8_t *state = (uint8_t *)xcalloc(length, 1);
  uint32_t *rep_of = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)length);
  uint32_t *member_count = (uint32_t *)xcalloc(length, sizeof(uint32_t));
  size_t b0 = 0;
  while (b0 < np) {
    size_t b1 = b0;
    while (b1 < np && (pairs[b1] >> 32) == (pairs[b0] >> 32)) ++b1;
    for (size_t i = b0; i < b1; ++i) {
      uint32_t c = (uint32_t)pairs[i];
      if (c < half) {
        state[c] = ST_NON_CLUSTERING;
      } else {
        for (uint32_t k = 0; k < L; ++k)
          if (db[c - half + k] == p->delimiter) {
            state[c] = ST_NON_CLUSTERING;
            break;
          }
      }
    }
    for (size_t i = b0; i < b1; ++i) {
      uint32_t r = (uint32_t)pairs[i];
      if (state[r] != ST_UNSET) continue;
      state[r] = ST_REP;
      for (size_t j = i + 1; j < b1; ++j) {
        uint32_t m = (uint32_t)pairs[j];
        if (state[m] != ST_UNSET) continue;
        if (gzo_distance(p, db, r, db, m) <= p->max_member_distance) {
          state[m] = ST_MEMBER;
          rep_of[m] = r;
        }
      }
    }
    b0 = b1;
  }
  for (size_t i = 0; i < np; ++i) {
    uint32_t c = (uint32_t)pairs[i];
    if (state[c] == ST_MEMBER) ++member_count[rep_of[c]];
  }

  /* 3. split into representatives, members and the residual index
   *    (:207-316) */
  uint64_t *nc_pairs = (uint64_t *)xmalloc(sizeof(uint64_t) * (np ? np : 1));
  uint64_t *rep_pairs = (uint64_t *)xmalloc(sizeof(uint64_t) * (np ? np : 1));
  size_t nnc = 0, nrep = 0, nmem = 0;
  uint32_t *cluster_of = rep_of; /* reuse: rep position -> cluster id */
  for (size_t i = 0; i < np; ++i) {
    uint32_t c = (uint32_t)pairs[i];
    if (state[c] == ST_REP && member_count[c] > 0) {
      rep_pairs[nrep++] = pairs[i];
    } else if (state[c] == ST_MEMBER) {
      ++nmem;
    } else {
      nc_pairs[nnc++] = pairs[i];
    }
  }
  /* cluster ids in (hash, position) order */
  uint32_t *rep_cluster = (uint32_t *)xmalloc(sizeof(uint32_t) * (nrep ? nrep : 1));
  for (size_t i = 0; i < nrep; ++i) rep_cluster[i] = (uint32_t)i;
  /* members must be looked up by representative -> cluster id; store the
   * id at the representative position in a side table. */
  uint32_t *pos_cluster = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)length);
  for (size_t i = 0; i < nrep; ++i) pos_cluster[(uint32_t)rep_pairs[i]] = (uint32_t)i;
  uint32_t *member_offsets = (uint32_t *)xcalloc(nrep + 1, sizeof(uint32_t));
  for (size_t i = 0; i < np; ++i) {
    uint32_t c = (uint32_t)pairs[i];
    if (state[c] == ST_MEMBER) ++member_offsets[pos_cluster[cluster_of[c]] + 1];
  }
  for (size_t i = 0; i < nrep; ++i) member_offsets[i + 1] += member_offsets[i];
  uint32_t *member_fill = (uint32_t *)xcalloc(nrep + 1, sizeof(uint32_t));
  uint32_t *member_positions = (uint32_t *)xmalloc(sizeof(uint32_t) * (nmem ? nmem : 1));
  /* members in database-position order within each cluster */
  {
    uint32_t *order = (uint32_t *)xmalloc(sizeof(uint32_t) * (nmem ? nmem : 1));
    size_t k = 0;
    for (size_t i = 0; i < np; ++i) {
      uint32_t c = (uint32_t)pairs[i];
      if (state[c] == ST_MEMBER) order[k++] = c;
    }
    /* pairs are (hash, position)-sorted and a member shares its
     * representative's hash, so members of one cluster already appear in
     * position order */
    for (size_t i = 0; i < nmem; ++i) {
      uint32_t c = order[i];
      uint32_t cid = pos_cluster[cluster_of[c]];
      member_positions[member_offsets[cid] + member_fill[cid]++] = c;
    }
    free(order);
  }

  csr_from_pairs(nc_pairs, nnc, &x->arr[0], &x->len[0], &x->arr[1],
                 &x->arr[2]);
  x->len[1] = x->len[0] + 1;
  x->len[2] = nnc;
  {
    uint32_t *rk, *ro, *rv;
    size_t nrk;
    csr_from_pairs(rep_pairs, nrep, &rk, &nrk, &ro, &rv);
    x->arr[3] = rk;
    x->len[3] = nrk;
    x->arr[4] = ro;
    x->len[4] = nrk + 1;
    x->arr[5] = rep_cluster;
    x->len[5] = nrep;
    x->arr[6] = rv;
    x->len[6] = nrep;
  }
  x->arr[7] = member_offsets;
  x->len[7] = nrep + 1;
  x->arr[8] = member_positions;
  x->len[8] = nmem;

  free(member_fill);
  free(pos_cluster);
  free(nc_pairs);
  free(rep_pairs);
  free(state);
  free(rep_of);
  free(member_count);
  free(pairs);
  return x;
}

void gzo_db_index_free(gzo_db_index *x) {
  if (!x) return;
  for (int i = 0; i < 9; ++i) free(x->arr[i]);
  free(x);
}

size_t gzo_db_index_array(const gzo_db_index *x, int which,
                          const uint32_t **data) {
  if (which < 0 || which > 8) {
    *data = NULL;
    return 0;
  }
  *data = x->arr[which];
  return x->len[which];
}

/* lookup in a sorted key array: index or -1 */
static long find_key(const uint32_t *keys, size_t n, uint32_t key) {
  size_t lo = 0, hi = n;
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    if (keys[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < n && keys[lo] == key) ? (long)lo : -1;
}

/* ------------------------------------------------------------------ */
/* Query hash-position lists.
 * Restates SeedSearcherGpuQueryParameters::Build
 * (src/seed_searcher_gpu_query_parameters.cpp:17-272): every position of a
 * delimiter-free stretch of at least L residues is hashed; a position is a
 * "check" position when the whole L window centred on it lies inside the
 * stretch; positions are grouped by hash.  Lists are ordered by hash and,
 * inside a list, check positions come first, each part in (query, position)
 * order (the reference's order depends on its thread scheduling and does
 * not change the seed set). */
struct gzo_query_lists {
  uint32_t *arr[5];
  size_t len[5];
};

typedef struct {
  uint32_t hash, nocheck, qid, pos;
} ent;

static const ent *qsort_ent_base; /* qsort has no context argument */

static int cmp_ent_order(const void *a, const void *b) {
  const ent *x = &qsort_ent_base[*(const uint32_t *)a];
  const ent *y = &qsort_ent_base[*(const uint32_t *)b];
  if (x->hash != y->hash) return x->hash < y->hash ? -1 : 1;
  if (x->nocheck != y->nocheck) return x->nocheck < y->nocheck ? -1 : 1;
  uint32_t ia = *(const uint32_t *)a, ib = *(const uint32_t *)b;
  return ia < ib ? -1 : (ia > ib ? 1 : 0);
}

gzo_query_lists *gzo_query_lists_build(const gzo_params *p,
                                       const uint8_t *queries,
                                       const uint32_t *offsets,
                                       const uint32_t *lengths,
                                       uint32_t number_queries) {
  const uint32_t L = (uint32_t)p->subsequence_length;
  size_t cap = 1024, n = 0;
  ent *e = (ent *)xmalloc(sizeof(ent) * cap);
  for (uint32_t qid = 0; qid < number_queries; ++qid) {
    const uint8_t *q = queries + offsets[qid];
    uint32_t qlen = lengths[qid];
    uint32_t off = 0;
    while (off < qlen) {
      uint32_t end = off;
      while (end < qlen && q[end] != p->delimiter) ++end;
      if (end - off >= L) {
        uint32_t cs = off + L / 2, ce = end - L / 2;
        for (uint32_t i = off; i < end; ++i) {
          uint32_t h, hl;
          if (!gzo_hash(p, q + i, &h, &hl)) {
            if (n == cap) {
              cap *= 2;
              e = (ent *)realloc(e, sizeof(ent) * cap);
              if (!e) abort();
            }
            e[n].hash = h;
            e[n].nocheck = !(cs <= i && i < ce);
            e[n].qid = qid;
            e[n].pos = i;
            ++n;
          }
        }
      }
      off = end + 1;
    }
  }
  /* order (hash, nocheck, entry index); entries are already in (query,
   * position) order, so the index keeps that order inside each part */
  qsort_ent_base = e;
  uint32_t *order = (uint32_t *)xmalloc(sizeof(uint32_t) * (n ? n : 1));
  for (size_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
  qsort(order, n, sizeof(uint32_t), cmp_ent_order);
  size_t nl = 0;
  for (size_t i = 0; i < n; ++i)
    if (i == 0 || e[order[i]].hash != e[order[i - 1]].hash) ++nl;
  gzo_query_lists *x = (gzo_query_lists *)xcalloc(1, sizeof(gzo_query_lists));
  x->arr[0] = (uint32_t *)xmalloc(4 * (nl ? nl : 1));
  x->arr[1] = (uint32_t *)xmalloc(4 * (nl + 1));
  x->arr[2] = (uint32_t *)xcalloc(nl ? nl : 1, 4);
  x->arr[3] = (uint32_t *)xmalloc(4 * (n ? n : 1));
  x->arr[4] = (uint32_t *)xmalloc(4 * (n ? n : 1));
  size_t l = 0;
  for (size_t i = 0; i < n; ++i) {
    const ent *t = &e[order[i]];
    if (i == 0 || t->hash != e[order[i - 1]].hash) {
      x->arr[0][l] = t->hash;
      x->arr[1][l] = (uint32_t)i;
      ++l;
    }
    if (!t->nocheck) ++x->arr[2][l - 1];
    x->arr[3][i] = t->qid;
    x->arr[4][i] = t->pos;
  }
  x->arr[1][nl] = (uint32_t)n;
  x->len[0] = nl;
  x->len[1] = nl + 1;
  x->len[2] = nl;
  x->len[3] = n;
  x->len[4] = n;
  free(order);
  free(e);
  return x;
}

void gzo_query_lists_free(gzo_query_lists *x) {
  if (!x) return;
  for (int i = 0; i < 5; ++i) free(x->arr[i]);
  free(x);
}

size_t gzo_query_lists_array(const gzo_query_lists *x, int which,
                             const uint32_t **data) {
  if (which < 0 || which > 4) {
    *data = NULL;
    return 0;
  }
  *data = x->arr[which];
  return x->len[which];
}

/* ------------------------------------------------------------------ */
/* Top-b merge.  Restates AlignerCommon::AddResults
 * (src/aligner_common.h:147-274) with AlignmentComp / IsContained
 * (src/aligner_common.cpp:12-68) and DatabaseChunk::GetId
 * (src/database_chunk.h:226-253).  The per-subject start list reproduces
 * the reference exactly: it is searched by database start but stores the
 * query start, and std::lower_bound is restated step for step. */
static int alignment_comp(const gzo_result *a, const gzo_result *b) {
  if (a->score > b->score) return 1;
  if (a->score < b->score) return -1;
  uint32_t aq = a->end_q - a->start_q, bq = b->end_q - b->start_q;
  if (aq > bq) return 1;
  if (aq < bq) return -1;
  uint32_t as = a->end_d - a->start_d, bs = b->end_d - b->start_d;
  if (as > bs) return 1;
  if (as < bs) return -1;
  return (a->start_d < b->start_d) ? 1 : -1;
}

static int is_contained(const gzo_result *a, const gzo_result *b) {
  return (a->start_q == b->start_q && a->start_d == b->start_d) ||
         (a->end_q == b->end_q && a->end_d == b->end_d) ||
         (a->start_q <= b->start_q && b->end_q <= a->end_q &&
          a->start_d <= b->start_d && b->end_d <= a->end_d);
}

static uint32_t subject_of(const uint32_t *db_offsets, uint32_t nseq,
                           uint32_t db_length, uint32_t position) {
  if (db_offsets[nseq - 1] <= position && position < db_length)
    return nseq - 1;
  /* largest i with offsets[i] <= position */
  uint32_t lo = 0, hi = nseq;
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (db_offsets[mid] <= position)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo == 0 ? 0xFFFFFFFFu : lo - 1;
}

/* stable merge sort by alignment_comp > 0 (descending) */
static void sort_results(gzo_result *r, size_t n, gzo_result *tmp) {
  if (n < 2) return;
  size_t h = n / 2;
  sort_results(r, h, tmp);
  sort_results(r + h, n - h, tmp);
  size_t i = 0, j = h, k = 0;
  while (i < h && j < n) {
    /* take right only when it is strictly greater than left */
    if (alignment_comp(&r[j], &r[i]) > 0)
      tmp[k++] = r[j++];
    else
      tmp[k++] = r[i++];
  }
  while (i < h) tmp[k++] = r[i++];
  while (j < n) tmp[k++] = r[j++];
  memcpy(r, tmp, sizeof(gzo_result) * n);
}

typedef struct {
  uint32_t result_id, position;
} start_pos;

/* std::lower_bound with operator< on .position, step for step */
static size_t lower_bound_pos(const start_pos *a, size_t first, size_t last,
                              uint32_t value) {
  size_t len = last - first;
  while (len > 0) {
    size_t half = len / 2;
    size_t mid = first + half;
    if (a[mid].position < value) {
      first = mid + 1;
      len = len - half - 1;
    } else {
      len = half;
    }
  }
  return first;
}

/* chunk_id of `added` entries must already be set by the caller; results
 * of other chunks pass through.  Returns the new length of `results`
 * (capacity >= max_number_results). */
static size_t add_results_chunk(const gzo_params *p, int32_t chunk_id,
                                const uint32_t *db_offsets, uint32_t nseq,
                                uint32_t db_length, gzo_result *added,
                                size_t n_added, gzo_result *results,
                                size_t n_results) {
  const size_t max_results = (size_t)p->max_number_results;
  gzo_result *tmp = (gzo_result *)xmalloc(sizeof(gzo_result) * (n_added ? n_added : 1));
  sort_results(added, n_added, tmp);
  free(tmp);
  gzo_result *out = (gzo_result *)xmalloc(sizeof(gzo_result) * (max_results + 1));
  size_t n_out = 0;
  /* per-subject start lists, only for subjects touched here */
  typedef struct {
    uint32_t subject;
    size_t n;
    start_pos v[64];
  } subj_list;
  size_t cap_lists = 16, n_lists = 0;
  subj_list *lists = (subj_list *)xmalloc(sizeof(subj_list) * cap_lists);
  size_t ri = 0, ai = 0;
  while (n_out < max_results && (ai < n_added || ri < n_results)) {
    gzo_result a;
    if (ai == n_added) {
      a = results[ri++];
    } else if (ri == n_results ||
               alignment_comp(&results[ri], &added[ai]) < 0) {
      a = added[ai];
      a.chunk_id = chunk_id;
      a.subject_id = (int32_t)subject_of(db_offsets, nseq, db_length,
                                         added[ai].start_d);
      ++ai;
    } else {
      a = results[ri++];
    }
    if (a.chunk_id == chunk_id) {
      subj_list *sl = NULL;
      for (size_t k = 0; k < n_lists; ++k)
        if (lists[k].subject == (uint32_t)a.subject_id) {
          sl = &lists[k];
          break;
        }
      if (!sl) {
        if (n_lists == cap_lists) {
          cap_lists *= 2;
          lists = (subj_list *)realloc(lists, sizeof(subj_list) * cap_lists);
          if (!lists) abort();
        }
        sl = &lists[n_lists++];
        sl->subject = (uint32_t)a.subject_id;
        sl->n = 0;
      }
      if (sl->n < (size_t)p->max_number_one_subject_results && sl->n < 64) {
        size_t it = lower_bound_pos(sl->v, 0, sl->n, a.start_d);
        size_t ins = it;
        size_t it_end = lower_bound_pos(sl->v, it, sl->n, a.end_d);
        int added_ok = 1;
        for (; it != it_end; ++it) {
          const gzo_result *r = &out[sl->v[it].result_id];
          if (is_contained(r, &a)) {
            added_ok = 0;
            break;
          }
        }
        if (added_ok) {
          memmove(&sl->v[ins + 1], &sl->v[ins],
                  sizeof(start_pos) * (sl->n - ins));
          sl->v[ins].position = a.start_q;
          sl->v[ins].result_id = (uint32_t)n_out;
          ++sl->n;
          out[n_out++] = a;
        }
      }
    } else {
      out[n_out++] = a;
    }
  }
  memcpy(results, out, sizeof(gzo_result) * n_out);
  free(out);
  free(lists);
  return n_out;
}

size_t gzo_add_results(const gzo_params *p, const uint32_t *db_offsets,
                       uint32_t number_sequences, uint32_t db_length,
                       gzo_result *added, size_t n_added, gzo_result *results,
                       size_t n_results) {
  int32_t chunk = n_added ? added[0].chunk_id : 0;
  return add_results_chunk(p, chunk, db_offsets, number_sequences, db_length,
                           added, n_added, results, n_results);
}

/* ------------------------------------------------------------------ */
/* Seed search for one query hash list.  Restates
 * SeedSearcher::SearchFromClusteringSubsequences /
 * SearchFromNonClusteringSubsequences (src/seed_searcher.cpp:103-295),
 * which the GPU driver splits into the same seed set
 * (src/seed_searcher_gpu.cpp:186-537): representatives are tested against
 * check positions by distance (kept when <= distance_threshold); their
 * members are tested for check positions whose representative distance
 * minus max_member_distance (floored at 0) is <= distance_threshold, and
 * for every no-check position; the residual index seeds every position. */
typedef struct {
  uint32_t *qid, *q, *d;
  size_t n, cap;
} hit_buf;

static void hit_push(hit_buf *b, uint32_t qid, uint32_t q, uint32_t d) {
  if (b->n == b->cap) {
    b->cap = b->cap ? b->cap * 2 : 1024;
    b->qid = (uint32_t *)realloc(b->qid, 4 * b->cap);
    b->q = (uint32_t *)realloc(b->q, 4 * b->cap);
    b->d = (uint32_t *)realloc(b->d, 4 * b->cap);
    if (!b->qid || !b->q || !b->d) abort();
  }
  b->qid[b->n] = qid;
  b->q[b->n] = q;
  b->d[b->n] = d;
  ++b->n;
}

struct gzo_presearch {
  uint32_t number_queries;
  gzo_result **results;
  size_t *n_results;
  gzo_counters counters;
  hit_buf hits;
};

typedef struct {
  uint32_t qid, q, d;
} hit3;
static int cmp_hit3(const void *a, const void *b) {
  const hit3 *x = (const hit3 *)a, *y = (const hit3 *)b;
  if (x->qid != y->qid) return x->qid < y->qid ? -1 : 1;
  if (x->d != y->d) return x->d < y->d ? -1 : 1;
  if (x->q != y->q) return x->q < y->q ? -1 : 1;
  return 0;
}

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
                                 uint32_t query_begin, uint32_t query_end) {
  gzo_presearch *x = (gzo_presearch *)xcalloc(1, sizeof(gzo_presearch));
  x->number_queries = number_queries;
  x->results = (gzo_result **)xcalloc(number_queries, sizeof(gzo_result *));
  x->n_results = (size_t *)xcalloc(number_queries, sizeof(size_t));
  gzo_counters *ct = &x->counters;

  const uint32_t *lh = index->arr[0]; /* placeholders for readability */
  (void)lh;
  const uint32_t *nc_keys = index->arr[0], *nc_off = index->arr[1],
                 *nc_val = index->arr[2];
  const size_t n_nc_keys = index->len[0];
  const uint32_t *rep_keys = index->arr[3], *rep_off = index->arr[4],
                 *rep_cid = index->arr[5], *rep_pos = index->arr[6];
  const size_t n_rep_keys = index->len[3];
  const uint32_t *mem_off = index->arr[7], *mem_pos = index->arr[8];

  const uint32_t *l_hash = lists->arr[0], *l_off = lists->arr[1],
                 *l_nchk = lists->arr[2], *e_qid = lists->arr[3],
                 *e_pos = lists->arr[4];
  const size_t n_lists = lists->len[0];

  size_t cap_pass = 64;
  uint32_t *pass = (uint32_t *)xmalloc(4 * cap_pass);

#define IN_RANGE(qid) ((qid) >= query_begin && (qid) < query_end)
#define TRY_SEED(qid, qpos, dpos)                                           \
  do {                                                                      \
    const uint8_t *qs_ = queries + query_offsets[qid];                      \
    ++ct->ungapped_seeds;                                                   \
    int s_ = gzo_ungapped_with_trigger(p, qs_, (qpos), db, (dpos),          \
                                       ungapped_cutoffs[qid],               \
                                       gapped_triggers[qid]);               \
    if (s_ > gapped_triggers[qid]) hit_push(&x->hits, (qid), (qpos), (dpos)); \
  } while (0)

  for (size_t li = 0; li < n_lists; ++li) {
    const uint32_t h = l_hash[li];
    const uint32_t b = l_off[li], e = l_off[li + 1];
    const uint32_t nchk = l_nchk[li];
    if ((size_t)(e - b) > cap_pass) {
      cap_pass = e - b;
      pass = (uint32_t *)realloc(pass, 4 * cap_pass);
      if (!pass) abort();
    }
    if (p->clustering) {
      long rk = find_key(rep_keys, n_rep_keys, h);
      if (rk >= 0) {
        for (uint32_t r = rep_off[rk]; r < rep_off[rk + 1]; ++r) {
          const uint32_t rpos = rep_pos[r];
          const uint32_t cid = rep_cid[r];
          size_t npass = 0;
          for (uint32_t k = b; k < e; ++k) {
            const uint32_t qid = e_qid[k], qpos = e_pos[k];
            int dist = 0;
            if (k < b + nchk) {
              if (IN_RANGE(qid)) ++ct->distance_seeds;
              dist = gzo_distance(p, queries + query_offsets[qid], qpos, db,
                                  rpos);
              int lb = dist - p->max_member_distance;
              if (lb < 0) lb = 0;
              if (p->distance_threshold >= lb) pass[npass++] = k;
            } else {
              pass[npass++] = k;
            }
            if (p->distance_threshold >= dist && IN_RANGE(qid))
              TRY_SEED(qid, qpos, rpos);
          }
          if (npass) {
            for (uint32_t m = mem_off[cid]; m < mem_off[cid + 1]; ++m)
              for (size_t t = 0; t < npass; ++t) {
                const uint32_t k = pass[t];
                if (IN_RANGE(e_qid[k])) TRY_SEED(e_qid[k], e_pos[k], mem_pos[m]);
              }
          }
        }
      }
    }
    long nk = find_key(nc_keys, n_nc_keys, h);
    if (nk >= 0) {
      for (uint32_t v = nc_off[nk]; v < nc_off[nk + 1]; ++v)
        for (uint32_t k = b; k < e; ++k)
          if (IN_RANGE(e_qid[k])) TRY_SEED(e_qid[k], e_pos[k], nc_val[v]);
    }
  }
  free(pass);
#undef TRY_SEED

  /* sort survivors by (query, d, q) */
  {
    size_t n = x->hits.n;
    hit3 *t = (hit3 *)xmalloc(sizeof(hit3) * (n ? n : 1));
    for (size_t i = 0; i < n; ++i) {
      t[i].qid = x->hits.qid[i];
      t[i].q = x->hits.q[i];
      t[i].d = x->hits.d[i];
    }
    qsort(t, n, sizeof(hit3), cmp_hit3);
    for (size_t i = 0; i < n; ++i) {
      x->hits.qid[i] = t[i].qid;
      x->hits.q[i] = t[i].q;
      x->hits.d[i] = t[i].d;
    }
    free(t);
    ct->ungapped_hits = n;
  }

  /* per query: chain filter, gapped extension of both sides, merge
   * (src/aligner_gpu_presearch_thread.cpp:472-614, 898-1008) */
  size_t i0 = 0;
  const size_t nh = x->hits.n;
  uint32_t *cq = NULL, *cd = NULL;
  size_t ccap = 0;
  while (i0 < nh) {
    size_t i1 = i0;
    const uint32_t qid = x->hits.qid[i0];
    while (i1 < nh && x->hits.qid[i1] == qid) ++i1;
    size_t n = i1 - i0;
    if (n > ccap) {
      ccap = n;
      cq = (uint32_t *)realloc(cq, 4 * ccap);
      cd = (uint32_t *)realloc(cd, 4 * ccap);
      if (!cq || !cd) abort();
    }
    memcpy(cq, x->hits.q + i0, 4 * n);
    memcpy(cd, x->hits.d + i0, 4 * n);
    const uint8_t *qs = queries + query_offsets[qid];
    const uint32_t qlen = query_lengths[qid];
    size_t kept = gzo_chain_filter(p, qs, qlen, ungapped_cutoffs[qid], db, cq,
                                   cd, n);
    ct->chained_hits += kept;
    gzo_result *added = (gzo_result *)xmalloc(sizeof(gzo_result) * (kept ? kept : 1));
    for (size_t k = 0; k < kept; ++k) {
      int sc, p0, p1;
      uint64_t cells;
      gzo_result *r = &added[k];
      memset(r, 0, sizeof(*r));
      r->hit_q = cq[k];
      r->hit_d = cd[k];
      /* reverse from (q-1, d-1); start = seed + best offset */
      gzo_gapped_one_side(p, qs + cq[k] - 1, db + cd[k] - 1, 1,
                          p->gapped_cutoff, &sc, &p0, &p1, &cells);
      r->score = sc;
      r->start_q = cq[k] - 1 + (uint32_t)p0;
      r->start_d = cd[k] - 1 + (uint32_t)p1;
      ct->gapped_cells += cells;
      /* forward from (q, d); end = seed + best offset (inclusive), the
       * convention of the GPU driver (src/aligner_gpu_presearch_thread.cpp:
       * 957-962) and of BuildResults
       * (src/aligner_build_results_thread.h:152-154) */
      gzo_gapped_one_side(p, qs + cq[k], db + cd[k], 0, p->gapped_cutoff, &sc,
                          &p0, &p1, &cells);
      r->score += sc;
      r->end_q = cq[k] + (uint32_t)p0;
      r->end_d = cd[k] + (uint32_t)p1;
      ct->gapped_cells += cells;
      ct->gapped_extensions += 2;
    }
    gzo_result *res = (gzo_result *)xmalloc(sizeof(gzo_result) * ((size_t)p->max_number_results + 1));
    size_t nres = add_results_chunk(p, 0, db_offsets, number_sequences,
                                    db_length, added, kept, res, 0);
    x->results[qid] = res;
    x->n_results[qid] = nres;
    free(added);
    i0 = i1;
  }
  free(cq);
  free(cd);
  return x;
}

void gzo_presearch_free(gzo_presearch *x) {
  if (!x) return;
  for (uint32_t i = 0; i < x->number_queries; ++i) free(x->results[i]);
  free(x->results);
  free(x->n_results);
  free(x->hits.qid);
  free(x->hits.q);
  free(x->hits.d);
  free(x);
}

size_t gzo_presearch_results(const gzo_presearch *x, uint32_t query_id,
                             const gzo_result **results) {
  if (query_id >= x->number_queries) {
    *results = NULL;
    return 0;
  }
  *results = x->results[query_id];
  return x->n_results[query_id];
}

void gzo_presearch_counters(const gzo_presearch *x, gzo_counters *out) {
  *out = x->counters;
}

size_t gzo_presearch_hits(const gzo_presearch *x, const uint32_t **qid,
                          const uint32_t **q, const uint32_t **d) {
  *qid = x->hits.qid;
  *q = x->hits.q;
  *d = x->hits.d;
  return x->hits.n;
}

/* ---- six-frame translation (src/translator.cpp:20-142,
 * src/translated_dna_query.cpp:44-74, src/dna_sequence.h:28-42) ---- */

/* The standard genetic code, codons in ACGT order (first base slowest). */
static const char kCodonTable[] =
    "KNKNTTTTRSRSIIMIQHQHPPPPRRRRLLLLEDEDAAAAGGGGVVVV*Y*YSSSS*CWCLFLF";
/* Protein code = index in this string (ProteinType regular letters, then
 * the ambiguous ones, then the unknown letter). */
static const char kProteinLetters[] = "ARNDCQEGHILKMFPSTWYVBJZ*X";

static int base_index(char c) {
  switch (c) {
    case 'A': return 0;
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    default: return -1;  /* the codon table is case sensitive */
  }
}

static char complement(char c) {
  switch (c) {
    case 'A': case 'a': return 'T';
    case 'C': case 'c': return 'G';
    case 'G': case 'g': return 'C';
    case 'T': case 't': return 'A';
    default: return 'N';
  }
}

static uint8_t protein_code(char letter) {
  for (uint8_t i = 0; kProteinLetters[i]; ++i)
    if (kProteinLetters[i] == letter) return i;
  return 24;
}

/* Translator::Translate keeps a "stopped" flag that is never set, so
 * every codon found in the table is translated and every other codon
 * becomes the unknown letter. */
static uint8_t codon_code(char a, char b, char c) {
  const int x = base_index(a), y = base_index(b), z = base_index(c);
  if (x < 0 || y < 0 || z < 0) return protein_code('X');
  return protein_code(kCodonTable[x * 16 + y * 4 + z]);
}

uint32_t gzo_translated_length(uint32_t length) {
  return length < 3 ? 2 : 7 + 6 * (length / 3);
}

uint32_t gzo_translate_query(const char *dna, uint32_t length, uint8_t delimiter,
                             uint8_t *out) {
  out[0] = delimiter;
  if (length < 3) {
    out[1] = delimiter;
    return 2;
  }
  char *rc = (char *)malloc(length);
  for (uint32_t i = 0; i < length; ++i) rc[i] = complement(dna[length - 1 - i]);
  const uint32_t base = length / 3;
  uint32_t o = 1;
  for (int frame = 0; frame < 6; ++frame) {
    const char *s = frame < 3 ? dna : rc;
    const uint32_t offset = (uint32_t)(frame % 3);
    uint32_t n = 0;
    for (uint32_t j = offset; j + 2 < length; j += 3, ++n)
      out[o + n] = codon_code(s[j], s[j + 1], s[j + 2]);
    o += n;
    if (n < base) out[o++] = delimiter;
    out[o++] = delimiter;
  }
  free(rc);
  return o;
}

/* ---- per-query Karlin-Altschul statistics ----
 * The sums below keep the reference's order of operations (serial, one
 * rounding per multiply and per add) so that the float results agree bit
 * for bit; the series for K is the one of Karlin & Altschul (1990) as the
 * reference's karlin.c evaluates it. */

#define GZO_KARLIN_ITER_MAX 100
#define GZO_SCORE_RANGE_MAX 11000

/* Robinson & Robinson background, ARNDCQEGHILKMFPSTWYV order
 * (src/statistics.cpp:154-176) */
static const double kRobinson[20] = {78.05, 51.29, 44.87, 53.64, 19.25, 42.64, 62.95,
                                     73.77, 21.99, 51.42, 90.19, 57.44, 22.43, 38.56,
                                     52.03, 71.20, 58.41, 13.30, 32.16, 64.41};

static int score_range_bad(int lo, int hi) {
  return lo >= 0 || hi <= 0 || lo < -10000 || hi > 1000 || hi - lo > GZO_SCORE_RANGE_MAX;
}

static long gcd_long(long a, long b) {
  long c;
  b = b < 0 ? -b : b;
  if (b > a) c = a, a = b, b = c;
  while (b != 0) {
    c = a % b;
    a = b;
    b = c;
  }
  return a;
}

/* lambda by bisection (karlin.c BlastKarlinLambdaBis) */
static double lambda_bisect(const double *sp, int lo, int hi) {
  if (score_range_bad(lo, hi)) return -1.0;
  double lambda = 0.0, up = 0.5, sum, x0, x1;
  for (;;) {
    up *= 2;
    x0 = exp(up);
    x1 = pow(x0, lo - 1);
    sum = 0.0;
    if (x1 > 0.0) {
      for (int i = lo; i <= hi; ++i) sum += sp[i] * (x1 *= x0);
    } else {
      for (int i = lo; i <= hi; ++i) sum += sp[i] * exp(up * i);
    }
    if (sum >= 1.0) break;
    lambda = up;
  }
  for (int j = 0; j < 17; ++j) {
    const double mid = (lambda + up) / 2.0;
    x0 = exp(mid);
    x1 = pow(x0, lo - 1);
    sum = 0.0;
    if (x1 > 0.0) {
      for (int i = lo; i <= hi; ++i) sum += sp[i] * (x1 *= x0);
    } else {
      for (int i = lo; i <= hi; ++i) sum += sp[i] * exp(mid * i);
    }
    if (sum > 1.0)
      up = mid;
    else
      lambda = mid;
  }
  return (lambda + up) / 2.0;
}

/* lambda by Newton-Raphson from 0.5 (karlin.c BlastKarlinLambdaNR) */
static double lambda_newton(const double *sp, int lo, int hi) {
  if (score_range_bad(lo, hi)) return -1.0;
  double lambda = 0.5;
  for (int j = 0; j < 20; ++j) {
    double sum = -1.0, slope = 0.0;
    if (lambda < 0.01) break;
    const double x0 = exp(lambda);
    double x1 = pow(x0, lo - 1);
    if (x1 == 0.0) break;
    for (int i = lo; i <= hi; ++i) {
      const double t = sp[i] * (x1 *= x0);
      sum += t;
      slope += t * i;
    }
    const double step = sum / slope;
    lambda -= step;
    if (fabs(step / lambda) < 1.0e-5) {
      if (lambda > 1.0e-5) return lambda;
      break;
    }
  }
  return lambda_bisect(sp, lo, hi);
}

/* relative entropy H (karlin.c BlastKarlinLtoH) */
static double entropy(const double *sp, int lo, int hi, double lambda) {
  if (lambda < 0.0 || score_range_bad(lo, hi)) return -1.0;
  const double etolam = exp(lambda);
  double etolami = pow(etolam, lo - 1), av = 0.0;
  if (etolami > 0.0) {
    for (int s = lo; s <= hi; ++s) av += sp[s] * s * (etolami *= etolam);
  } else {
    for (int s = lo; s <= hi; ++s) av += sp[s] * s * exp(lambda * s);
  }
  return lambda * av;
}

/* K from lambda and H (karlin.c BlastKarlinLHtoK): the series
 * sum_j (1/j) [E(exp(lambda S_j); S_j < 0) + P(S_j >= 0)] over the j-fold
 * convolutions of the score distribution, closed with a geometric tail. */
static double karlin_k(const double *sp, int low, int high, double lambda, double H) {
  if (lambda <= 0.0 || H <= 0.0) return -1.0;
  const int range = high - low;
  const double av = H / lambda;
  const double etolam = exp(lambda);
  if (low == -1 || high == 1) return av * (1.0 - 1.0 / etolam);
  double sumlimit = 0.01;
  const int iter = GZO_KARLIN_ITER_MAX;
  if (iter * range + 1 > GZO_KARLIN_ITER_MAX * GZO_SCORE_RANGE_MAX + 1) return -1.0;
  double *cur = (double *)calloc((size_t)iter * range + 1, sizeof(double));
  double *nxt = (double *)calloc((size_t)iter * range + 1, sizeof(double));
  const double *p = sp + low;  /* p[u] = probability of score low + u */
  double sum = 1.0, oldsum = 1.0, oldsum2 = 1.0, total = 0.0, K;
  int lo = 0, hi = 0, j = 0;
  cur[0] = 1.0;
  while (j < iter && sum > sumlimit) {
    lo += low;
    hi += high;
    const int top = hi - lo;
    /* next distribution: entry k takes u = first..last in increasing order */
    for (int k = 0; k <= top; ++k) {
      const int first = range - (top - k) > 0 ? range - (top - k) : 0;
      const int last = k < range ? k : range;
      double s = 0.0;
      for (int u = first; u <= last; ++u) s += cur[k - u] * p[u];
      nxt[k] = s;
    }
    double etolami = pow(etolam, lo - 1);
    int i = lo, idx = 0;
    double s = 0.0;
    for (; i != 0; ++i, ++idx) {
      etolami *= etolam;
      s += nxt[idx] * etolami;
    }
    for (; i <= hi; ++i, ++idx) s += nxt[idx];
    oldsum2 = oldsum;
    oldsum = s;
    double *t = cur;
    cur = nxt;
    nxt = t;
    sum = s / ++j;
    total += sum;
  }
  const double ratio = oldsum / oldsum2;
  if (ratio >= (1.0 - sumlimit * 0.001)) {
    K = -1.0;
  } else {
    sumlimit *= 0.01;
    while (sum > sumlimit) {
      oldsum *= ratio;
      total += sum = oldsum / ++j;
    }
    long delta = -low;
    for (int i = 1; i <= range && delta > 1; ++i)
      if (p[i] != 0.0) delta = gcd_long(delta, i);
    if (delta * etolam > 0.05) {
      const double etolami = pow(etolam, -delta);
      K = delta * exp(-2.0 * total) / (av * (1.0 - etolami));
    } else {
      K = -delta * exp(-2.0 * total) / (av * (exp(-delta * lambda) - 1));
    }
  }
  free(cur);
  free(nxt);
  return K;
}

int gzo_query_karlin(const gzo_params *p, const uint8_t *seq, uint32_t length,
                     float ungapped_bits, float trigger_bits, float *lambda, float *k,
                     float *h, int32_t *cutoff, int32_t *trigger) {
  const int n = p->number_letters;
  const int max_code = n - 1, max_regular = 19;
  double bg[64], freq[64];
  /* background: Robinson, normalised (Statistics::Statistics and Normalize) */
  double sum = 0.0;
  for (int c = 0; c <= max_code; ++c) bg[c] = c < 20 ? kRobinson[c] : 0.0;
  for (int c = 0; c <= max_code; ++c) sum += bg[c];
  for (int c = 0; c <= max_code; ++c) {
    bg[c] /= sum;
    bg[c] *= 1.0;
  }
  /* query composition with a pseudo-count for absent letters
   * (ComposeSequenceFrequency, then Normalize) */
  for (int c = 0; c <= max_code; ++c) freq[c] = 0.0;
  for (uint32_t i = 0; i < length; ++i)
    if (seq[i] <= max_regular) ++freq[seq[i]];
  for (int c = 0; c <= max_code; ++c)
    if (freq[c] < 1.0) ++freq[c];
  sum = 0.0;
  for (int c = 0; c <= max_code; ++c) sum += freq[c];
  for (int c = 0; c <= max_code; ++c) {
    freq[c] /= sum;
    freq[c] *= 1.0;
  }
  /* score probabilities (CalculateScoreProbabilities) */
  int lo = p->score_matrix[0], hi = p->score_matrix[0];
  for (int i = 0; i < n * n; ++i) {
    lo = p->score_matrix[i] < lo ? p->score_matrix[i] : lo;
    hi = p->score_matrix[i] > hi ? p->score_matrix[i] : hi;
  }
  double *sp0 = (double *)calloc((size_t)(hi - lo + 1), sizeof(double));
  double *sp = sp0 - lo;
  for (int c1 = 0; c1 <= max_code; ++c1)
    for (int c2 = 0; c2 <= max_code; ++c2)
      sp[p->score_matrix[c1 * n + c2]] += freq[c1] * bg[c2];
  double ssum = 0.0;
  for (int i = lo; i <= hi; ++i)
    if (sp[i] > 0.0) ssum += sp[i];
  for (int i = lo; i <= hi; ++i)
    if (sp[i] > 0.0) sp[i] /= ssum;
  /* BlastKarlinBlkCalc: each parameter rounded to float before the next */
  const float l = (float)lambda_newton(sp, lo, hi);
  const float hh = (float)entropy(sp, lo, hi, l);
  const float kk = (float)karlin_k(sp, lo, hi, l, hh);
  free(sp0);
  *lambda = l;
  *k = kk;
  *h = hh;
  /* NormalizedCutoff2NominalCutoff and Normalized2Nominal in float */
  const float ln2 = (float)log(2.0);
  const float c = (ungapped_bits * ln2) / l;
  const float t = (trigger_bits * ln2 + logf(kk)) / l;
  *cutoff = (int32_t)floorf(c);
  *trigger = (int32_t)floorf(t);
  return 0;
}

/* ---- SEG (Wootton & Federhen) as the reference's ext/seg implements it ----
 * Parameters: window 12, low cut 2.2 bits, high cut 2.5 bits, window
 * entropies keyed by the window's first position, trimming over at most
 * 100 shorter lengths (ext/seg/src/seg.cpp:58-76). */

#define SEG_WINDOW 12
#define SEG_LOW_CUT 2.2
#define SEG_HIGH_CUT 2.5
#define SEG_MAX_TRIM 100
#define SEG_LN_FACT_SIZE 65536

static double seg_ln_fact[SEG_LN_FACT_SIZE];
static double seg_entropy12[SEG_WINDOW + 1];
static int seg_ready = 0;

double gzo_ln_factorial6(uint32_t n) {
  /* ln(n!) from the long-double log-gamma, rounded to 6 decimals through
   * its decimal text, which is how the reference's table is written */
  char text[64];
  snprintf(text, sizeof text, "%.6Lf", n < 2 ? 0.0L : lgammal((long double)n + 1.0L));
  return strtod(text, NULL);
}

static void seg_init(void) {
  if (seg_ready) return;
  for (uint32_t n = 0; n < SEG_LN_FACT_SIZE; ++n) seg_ln_fact[n] = gzo_ln_factorial6(n);
  const double w = SEG_WINDOW, ln2 = log(2.0);
  for (int i = 1; i <= SEG_WINDOW; ++i) {
    const double x = i / w;
    seg_entropy12[i] = -x * log(x) / ln2;
  }
  seg_ready = 1;
}

/* index of an amino-acid letter SEG counts, or -1 (upper case only) */
static int seg_class(char c) {
  static const char *aa = "ACDEFGHIKLMNPQRSTVWY";
  for (int i = 0; i < 20; ++i)
    if (aa[i] == c) return i;
  return -1;
}

/* counts of the window's letters, sorted in decreasing order, 0-terminated */
static int seg_state(const char *s, int n, int *state) {
  int comp[20] = {0};
  for (int i = 0; i < n; ++i) {
    const int k = seg_class(s[i]);
    if (k >= 0) ++comp[k];
  }
  int m = 0;
  for (int k = 0; k < 20; ++k)
    if (comp[k]) state[m++] = comp[k];
  for (int a = 1; a < m; ++a)  /* insertion sort, decreasing */
    for (int b = a; b > 0 && state[b - 1] < state[b]; --b) {
      const int t = state[b];
      state[b] = state[b - 1];
      state[b - 1] = t;
    }
  for (int k = m; k <= 20; ++k) state[k] = 0;
  return m;
}

static double seg_entropy(const int *state) {
  int total = 0, m = 0;
  for (; state[m]; ++m) total += state[m];
  double ent = 0.0;
  if (total == SEG_WINDOW) {
    for (int i = 0; i < m; ++i) ent += seg_entropy12[state[i]];
    return ent;
  }
  if (total == 0) return 0.0;
  const double r = 1.0 / (double)total;
  for (int i = 0; i < m; ++i) {
    const double v = state[i];
    ent += v * log(v * r);
  }
  return -ent * r / log(2.0);
}

/* entropy of the window keyed by position i of a sequence of n letters:
 * the window starting at i, or the last full window past n - 12 */
static double seg_h(const char *s, int n, int i) {
  int state[21];
  const int start = i < n - SEG_WINDOW ? i : n - SEG_WINDOW;
  seg_state(s + start, SEG_WINDOW, state);
  return seg_entropy(state);
}

/* ln of the probability of the window's composition
 * (Seg::GetProbability: LnAss + LnPerm - n ln 20) */
static double seg_probability(const int *state, int total) {
  double ass = seg_ln_fact[20];
  if (state[0] != 0) {
    int left = 20, run = 1, prev = state[0];
    for (int i = 1; i < 20; ++i) {
      const int v = state[i];
      if (v == prev) {
        ++run;
      } else {
        left -= run;
        ass -= seg_ln_fact[run];
        if (v == 0) {
          run = left;
          break;
        }
        run = 1;
      }
      prev = v;
    }
    ass -= seg_ln_fact[run];
  }
  double perm = seg_ln_fact[total];
  for (int i = 0; state[i] != 0; ++i) perm -= seg_ln_fact[state[i]];
  return ass + perm - (double)total * log(20.0);
}

/* Seg::Trim over s[0..n): the sub-window of length > max(1, n - 100) with
 * the least probable composition (first found wins) */
static void seg_trim(const char *s, int n, int *left, int *right) {
  int best_left = 0, best_right = n - 1;
  int min_length = 1;
  if (n - SEG_MAX_TRIM > min_length) min_length = n - SEG_MAX_TRIM;
  double best = 1.0;
  int state[21];
  for (int len = n; len > min_length; --len) {
    for (int i = 0; i + len <= n; ++i) {
      seg_state(s + i, len, state);
      const double p = seg_probability(state, len);
      if (p < best) {
        best = p;
        best_left = i;
        best_right = len + i - 1;
      }
    }
  }
  *left += best_left;
  *right -= n - best_right - 1;
}

/* Seg::MakeSeqments over s[0..n) (recursing into the part left of a
 * trimmed segment), marking every segment in mask */
static void seg_segments(const char *s, int n, unsigned char *mask) {
  if (n < SEG_WINDOW) return;
  int left_limit = 0;
  for (int i = 0; i <= n - 1; ++i) {
    if (seg_h(s, n, i) > SEG_LOW_CUT) continue;
    int lo = i;
    while (lo >= left_limit && seg_h(s, n, lo) <= SEG_HIGH_CUT) --lo;
    const int left_i = lo + 1;
    int hi = i;
    while (hi <= n - 1 && seg_h(s, n, hi) <= SEG_HIGH_CUT) ++hi;
    const int right_i = hi - 1;
    int left_end = left_i, right_end = right_i;
    seg_trim(s + left_end, right_end - left_end + 1, &left_end, &right_end);
    if (i < left_end) seg_segments(s + left_i, left_end - left_i, mask + left_i);
    for (int k = left_end; k <= right_end; ++k) mask[k] = 1;
    i = right_i < right_end ? right_i : right_end;
    left_limit = i + 1;
  }
}

int gzo_seg_mask(const char *seq, uint32_t length, char *out) {
  if (length < SEG_WINDOW) return 1;
  seg_init();
  unsigned char *mask = (unsigned char *)calloc(length, 1);
  seg_segments(seq, (int)length, mask);
  for (uint32_t i = 0; i < length; ++i) {
    const char c = seq[i];
    out[i] = mask[i] ? 'x' : (c >= 'a' && c <= 'z' ? (char)(c - 'a' + 'A') : c);
  }
  free(mask);
  return 0;
}

uint32_t gzo_translate_query_seg(const char *dna, uint32_t length, uint8_t delimiter,
                                 uint8_t *out) {
  const uint32_t n = gzo_translate_query(dna, length, delimiter, out);
  if (length < 3) return n;
  const uint32_t slot = length / 3 + 1;
  char letters[SEG_LN_FACT_SIZE], masked[SEG_LN_FACT_SIZE];
  for (int f = 0; f < 6; ++f) {
    uint8_t *q = out + 1 + f * slot;
    uint32_t m = 0;
    while (m < slot && q[m] != delimiter) ++m;
    if (m >= SEG_LN_FACT_SIZE) return 0;
    for (uint32_t i = 0; i < m; ++i) letters[i] = kProteinLetters[q[i]];
    if (gzo_seg_mask(letters, m, masked) != 0) {
      for (uint32_t i = 0; i < m; ++i) q[i] = protein_code('X');
    } else {
      for (uint32_t i = 0; i < m; ++i) q[i] = masked[i] == 'x' ? protein_code('X')
                                                                : protein_code(masked[i]);
    }
  }
  return n;
}

void gzo_protein_query_seg(const char *letters, uint32_t length, uint8_t delimiter,
                           uint8_t *out) {
  memset(out, 0, length + 2);
  out[0] = delimiter;
  char *masked = (char *)malloc(length + 1);
  if (gzo_seg_mask(letters, length, masked) == 0) {
    for (uint32_t i = 0; i < length; ++i)
      out[1 + i] = masked[i] == 'x' ? protein_code('X') : protein_code(masked[i]);
    out[length + 1] = delimiter;
  }
  free(masked);
}

/* ---- statistics of the final hit table ---- */

uint64_t gzo_search_space(uint64_t query_length, uint64_t db_length, uint64_t db_sequences,
                          float lambda, float k, double alpha, double beta) {
  /* the length adjustment: the BLAST fixed point of
   * ell = alpha/lambda (ln K + ln((m - ell)(n - N ell))) + beta */
  uint64_t adjust = 0;
  const double m = (double)query_length, n = (double)db_length, N = (double)db_sequences;
  const double log_k = logf(k);
  const double a_l = alpha / lambda;
  const double a = N, mb = m * N + n;
  const double c = n * m - (m > n ? m : n) / k;
  if (c >= 0) {
    double e, e_min = 0, e_max = 2 * c / (mb + sqrt(mb * mb - 4 * a * c)), ss, e_next = 0.0;
    int converged = 0;
    for (int i = 0; i < 20; ++i) {
      e = e_next;
      ss = (m - e) * (n - N * e);
      const double e_bar = a_l * (log_k + log(ss)) + beta;
      if (e_bar >= e) {
        e_min = e;
        if (e_bar - e_min <= 1.0) {
          converged = 1;
          break;
        }
        if (e_min >= e_max) break;
      } else {
        e_max = e;
      }
      if (e_min <= e_bar && e_bar <= e_max)
        e_next = e_bar;
      else
        e_next = i == 0 ? e_max : (e_min + e_max) / 2;
    }
    adjust = (uint64_t)(int)e_min;
    if (converged) {
      e = ceil(e_min);
      if (e <= e_max) {
        ss = (m - e) * (n - N * e);
        if (a_l * (log_k + log(ss)) + beta > e) adjust = (uint64_t)(int)e;
      }
    }
  }
  const uint64_t effective_db = db_length - db_sequences * adjust;
  return effective_db * (query_length - adjust);
}

double gzo_evalue(int32_t score, uint64_t search_space, float lambda, float k) {
  /* the search space times K is a float product */
  const float sk = (float)search_space * k;
  return sk * exp(-1.0 * score * lambda);
}

float gzo_bit_score(int32_t score, float lambda, float k) {
  return ((float)score * lambda - logf(k)) / (float)log(2.0);
}

uint32_t gzo_translated_real_start(uint32_t position, uint32_t dna_length) {
  const uint32_t base = dna_length / 3 + 1;
  const uint32_t f = (position - 1) / base;
  if (f < 3) return ((position % base) - 1) * 3 + f + 1;
  return dna_length - (((position % base) - 1) * 3 + f - 2) + 1;
}

uint32_t gzo_translated_real_end(uint32_t position, uint32_t dna_length) {
  const uint32_t base = dna_length / 3 + 1;
  const uint32_t f = (position - 1) / base;
  return f < 3 ? gzo_translated_real_start(position, dna_length) + 2
               : gzo_translated_real_start(position, dna_length) - 2;
}
