// gzb_hits.cu -- statistics of the final hit table (host code): the values
// AlignerCommon::WriteOutput (src/aligner_common.h:344-394) prints beside a
// result's alignment statistics, and the read coordinates of translated
// queries.
//
// The arithmetic keeps the reference's types and order, because the
// printed values depend on them: the gapped Karlin parameters are floats;
// the search space's length adjustment is BLAST's fixed-point iteration
// (Statistics::CalculateLengthAdjustment, src/statistics.cpp:56-122) with
// ln K taken in float; the E-value multiplies the search space by K in float
// before the double exponential (Nominal2EValue, :44-48); the normalized
// score is computed in float (Nominal2Normalized, :23-27).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ghostz_b200.h"
#include "gzb_common.h"

extern "C" int gzb_gapped_karlin_parameters(const char *matrix_name, int gap_open,
                                            int gap_extension, float *lambda, float *k,
                                            float *h, double *alpha, double *beta) {
  GZB_CHECK(matrix_name && lambda && k && h && alpha && beta, GZB_ERR_INVALID,
            "gzb_gapped_karlin_parameters: null argument");
  // Statistics::CalculateGappedKarlinParameters / CalculateAlphaBeta
  // (src/statistics.cpp:232-270): the published values for two matrices
  if (std::strcmp(matrix_name, "BLOSUM62") == 0 && gap_open == 11 && gap_extension == 1) {
    *lambda = 0.267f;
    *k = 0.041f;
    *h = 0.14f;
    *alpha = 1.9;
    *beta = -30;
    return GZB_OK;
  }
  if (std::strcmp(matrix_name, "PAM30") == 0 && gap_open == 9 && gap_extension == 1) {
    *lambda = 0.294f;
    *k = 0.11f;
    *h = 0.61f;
    *alpha = 0.48;
    *beta = -6;
    return GZB_OK;
  }
  return gzb::set_error(GZB_ERR_INVALID,
                        "no gapped Karlin parameters for %s with gap open %d, extension %d",
                        matrix_name, gap_open, gap_extension);
}

extern "C" uint64_t gzb_search_space(uint64_t query_length, uint64_t db_length,
                                     uint64_t db_sequences, float lambda, float k, double alpha,
                                     double beta) {
  uint64_t adjust = 0;
  const double m = (double)query_length, n = (double)db_length, N = (double)db_sequences;
  const double log_k = std::log(k);  // the float logarithm
  const double a_l = alpha / lambda;
  const double a = N, mb = m * N + n;
  const double c = n * m - (m > n ? m : n) / k;
  if (c >= 0) {
    double e_min = 0, e_max = 2 * c / (mb + std::sqrt(mb * mb - 4 * a * c)), e_next = 0.0;
    bool converged = false;
    for (int i = 0; i < 20; ++i) {
      const double e = e_next;
      const double space = (m - e) * (n - N * e);
      const double e_bar = a_l * (log_k + std::log(space)) + beta;
      if (e_bar >= e) {
        e_min = e;
        if (e_bar - e_min <= 1.0) {
          converged = true;
          break;
        }
        if (e_min >= e_max) break;
      } else {
        e_max = e;
      }
      e_next = (e_min <= e_bar && e_bar <= e_max) ? e_bar : (i == 0 ? e_max : (e_min + e_max) / 2);
    }
    adjust = (uint64_t)(int)e_min;
    if (converged) {
      const double e = std::ceil(e_min);
      if (e <= e_max && a_l * (log_k + std::log((m - e) * (n - N * e))) + beta > e)
        adjust = (uint64_t)(int)e;
    }
  }
  return (db_length - db_sequences * adjust) * (query_length - adjust);
}

extern "C" double gzb_evalue(int32_t score, uint64_t search_space, float lambda, float k) {
  const float sk = (float)search_space * k;
  return sk * std::exp(-1.0 * score * lambda);
}

extern "C" float gzb_bit_score(int32_t score, float lambda, float k) {
  return ((float)score * lambda - std::log(k)) / (float)std::log(2.0);
}

extern "C" uint32_t gzb_translated_real_start(uint32_t position, uint32_t dna_length) {
  const uint32_t base = dna_length / 3 + 1;
  const uint32_t f = (position - 1) / base;
  if (f < 3) return ((position % base) - 1) * 3 + f + 1;
  return dna_length - (((position % base) - 1) * 3 + f - 2) + 1;
}

extern "C" uint32_t gzb_translated_real_end(uint32_t position, uint32_t dna_length) {
  const uint32_t base = dna_length / 3 + 1;
  const uint32_t f = (position - 1) / base;
  return f < 3 ? gzb_translated_real_start(position, dna_length) + 2
               : gzb_translated_real_start(position, dna_length) - 2;
}

namespace {
// One record with the coordinates AlignerCommon::BuildResult leaves in a
// Result (src/aligner_common.h:326-340): the query's real start and end, the
// subject-relative database start and end.
struct FinalRow {
  gzb_alignment a;
  uint32_t q_start, q_end, d_start, d_end;
};

// AlignerCommon::AlignmentComp(...) > 0 (src/aligner_common.cpp:12-52): a
// comes first on a higher score, then a longer query span, then a longer
// subject span, then a smaller subject start; equal subject starts compare
// as "not first" both ways.
bool result_greater(const FinalRow &x, const FinalRow &y) {
  if (x.a.score != y.a.score) return x.a.score > y.a.score;
  const uint32_t xq = x.q_end - x.q_start, yq = y.q_end - y.q_start;
  if (xq != yq) return xq > yq;
  const uint32_t xs = x.d_end - x.d_start, ys = y.d_end - y.d_start;
  if (xs != ys) return xs > ys;
  return x.d_start < y.d_start;
}
}  // namespace

extern "C" int gzb_sort_alignments(uint32_t number_queries, uint32_t stride,
                                   const uint32_t *counts, gzb_alignment *alignments,
                                   uint32_t number_subjects, const uint32_t *db_offsets,
                                   const uint32_t *dna_lengths) {
  GZB_CHECK(number_queries == 0 || (counts && alignments && db_offsets), GZB_ERR_INVALID,
            "null argument");
  std::vector<FinalRow> rows;
  for (uint32_t q = 0; q < number_queries; ++q) {
    GZB_CHECK(counts[q] <= stride, GZB_ERR_INVALID, "query %u: %u results in rows of %u", q,
              counts[q], stride);
    gzb_alignment *row = alignments + (size_t)q * stride;
    rows.clear();
    for (uint32_t i = 0; i < counts[q]; ++i) {
      const gzb_alignment &a = row[i];
      GZB_CHECK(a.subject_id >= 0 && (uint32_t)a.subject_id < number_subjects, GZB_ERR_INVALID,
                "query %u: subject %d out of range", q, a.subject_id);
      FinalRow r;
      r.a = a;
      r.q_start = dna_lengths ? gzb_translated_real_start(a.start_q, dna_lengths[q]) : a.start_q;
      r.q_end = dna_lengths ? gzb_translated_real_end(a.end_q, dna_lengths[q]) : a.end_q;
      const uint32_t first = db_offsets[a.subject_id] - 1;
      r.d_start = a.start_d - first;
      r.d_end = a.end_d - first;
      rows.push_back(r);
    }
    std::sort(rows.begin(), rows.end(), result_greater);
    for (uint32_t i = 0; i < counts[q]; ++i) row[i] = rows[i].a;
  }
  return GZB_OK;
}

// The tabular lines of AlignerCommon::WriteOutput (src/aligner_common.h:
// 344-394): query and subject names, identity %, alignment length,
// mismatches, gap openings, query start and end (a read's bases for a
// translated query), subject start and end (1-based in the subject),
// E-value and normalized score, numbers as a C++ stream prints them (six
// significant digits).  The identity is 1 - (differences / length) with the
// division in float.  Rows with alignment_length 0 (results no build step
// filled) are skipped.
extern "C" int gzb_write_hit_table(uint32_t number_queries, uint32_t stride,
                                   const uint32_t *counts, const gzb_alignment *alignments,
                                   const char *const *query_names,
                                   const char *const *subject_names, uint32_t number_subjects,
                                   const uint32_t *db_offsets, uint64_t db_length,
                                   uint64_t db_sequences, const uint32_t *query_real_lengths,
                                   const uint32_t *dna_lengths, float lambda, float k,
                                   double alpha, double beta, char *out, uint64_t capacity,
                                   uint64_t *written) {
  GZB_CHECK(written && (number_queries == 0 || (counts && alignments && query_names &&
                                                subject_names && db_offsets &&
                                                query_real_lengths)),
            GZB_ERR_INVALID, "null argument");
  std::string text;
  char buf[160];
  for (uint32_t q = 0; q < number_queries; ++q) {
    GZB_CHECK(counts[q] <= stride, GZB_ERR_INVALID, "query %u: %u results in rows of %u", q,
              counts[q], stride);
    if (counts[q] == 0) continue;
    const uint64_t space =
        gzb_search_space(query_real_lengths[q], db_length, db_sequences, lambda, k, alpha, beta);
    for (uint32_t i = 0; i < counts[q]; ++i) {
      const gzb_alignment &a = alignments[(size_t)q * stride + i];
      if (a.alignment_length == 0) continue;
      GZB_CHECK(a.subject_id >= 0 && (uint32_t)a.subject_id < number_subjects, GZB_ERR_INVALID,
                "query %u: subject %d out of range", q, a.subject_id);
      const float diff = (float)(a.mismatches + a.gap_openings + a.gap_extensions);
      const double identity = (1.0 - (double)(diff / (float)a.alignment_length)) * 100;
      uint32_t sq = a.start_q, eq = a.end_q;
      if (dna_lengths) {
        sq = gzb_translated_real_start(sq, dna_lengths[q]);
        eq = gzb_translated_real_end(eq, dna_lengths[q]);
      }
      const uint32_t first = db_offsets[a.subject_id] - 1;
      text += query_names[q];
      text += '\t';
      text += subject_names[a.subject_id];
      snprintf(buf, sizeof(buf), "\t%g\t%u\t%u\t%u\t%u\t%u\t%u\t%u\t%g\t%g\n", identity,
               a.alignment_length, a.mismatches, a.gap_openings, sq, eq, a.start_d - first,
               a.end_d - first, gzb_evalue(a.score, space, lambda, k),
               (double)gzb_bit_score(a.score, lambda, k));
      text += buf;
    }
  }
  *written = text.size();
  if (!out) return GZB_OK;
  GZB_CHECK(capacity >= text.size(), GZB_ERR_INVALID, "hit table needs %llu bytes",
            (unsigned long long)text.size());
  memcpy(out, text.data(), text.size());
  return GZB_OK;
}
