// gzb_merge.cu -- the exchange step of a search whose database chunks are
// spread over GPUs: one chunk's per-query top-b lists merged into the
// running lists on the host, as the reference's AddResults merges each
// chunk's results (src/aligner_common.h:147-274).  Host code only.
//
// Why per-chunk lists suffice: AddResults filters a chunk's candidates
// (per-subject limit and containment) against that chunk's accepted
// candidates only -- results of other chunks pass unfiltered -- and walks
// them in their sorted order, so the candidates a chunk can contribute are
// the first max_number_results of its own filtered list, which is what the
// engine holds after gzb_engine_reset_results and one presearch of that
// chunk.  Merging those lists in chunk order therefore repeats the running
// merge exactly (ties included, since the two-way merge is the same).

#include <algorithm>
#include <cstring>

#include "ghostz_b200.h"
#include "gzb_common.h"

namespace {

// AlignerCommon::AlignmentComp (src/aligner_common.cpp:12-47): score, then
// query length, then database length, then the smaller database start; it
// never reports equality.
int alignment_comp(const gzb_result &a, const gzb_result &b) {
  if (a.score != b.score) return a.score > b.score ? 1 : -1;
  const uint32_t aq = a.end_q - a.start_q, bq = b.end_q - b.start_q;
  if (aq != bq) return aq > bq ? 1 : -1;
  const uint32_t as = a.end_d - a.start_d, bs = b.end_d - b.start_d;
  if (as != bs) return as > bs ? 1 : -1;
  return a.start_d < b.start_d ? 1 : -1;
}

// AlignerCommon::IsContained (src/aligner_common.cpp:54-68): b shares a's
// start or end, or lies inside a.
bool contained(const gzb_result &a, const gzb_result &b) {
  return (a.start_q == b.start_q && a.start_d == b.start_d) ||
         (a.end_q == b.end_q && a.end_d == b.end_d) ||
         (a.start_q <= b.start_q && b.end_q <= a.end_q && a.start_d <= b.start_d &&
          b.end_d <= a.end_d);
}

constexpr int kMaxResults = 32;  // max_number_results is at most 32

struct Start {
  uint32_t position, result;  // the reference keys the list by this position
};

struct SubjectStarts {
  int32_t subject;
  int n;
  Start starts[kMaxResults];  // ordered by position
};

// std::lower_bound's bisection over [from, n).  The list need not be sorted
// by the searched value (entries are inserted where their database start
// would go but keyed by their query start), so the probes must be the
// bisection's exactly, not a scan.
int first_not_below(const Start *v, int from, int n, uint32_t position) {
  int len = n - from;
  while (len > 0) {
    const int half = len >> 1, mid = from + half;
    if (v[mid].position < position) {
      from = mid + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return from;
}

// One query: `added` (n_added records of one chunk) merged into `row`
// (n_row records), at most b kept; returns the new count.  No allocation:
// every list is bounded by b <= 32.
uint32_t merge_row(const gzb_params &p, gzb_result *added, uint32_t n_added, gzb_result *row,
                   uint32_t n_row) {
  const uint32_t b = (uint32_t)p.max_number_results;
  // stable, best first (stable_sort with PresearchedResultGreaterScore):
  // insertion sort moves a record only past strictly worse ones
  for (uint32_t i = 1; i < n_added; ++i) {
    const gzb_result x = added[i];
    uint32_t j = i;
    while (j > 0 && alignment_comp(x, added[j - 1]) > 0) {
      added[j] = added[j - 1];
      --j;
    }
    added[j] = x;
  }
  const int32_t chunk = n_added ? added[0].chunk_id : -1;
  gzb_result out[kMaxResults];
  uint32_t n_out = 0;
  SubjectStarts subjects[kMaxResults];
  int n_subjects = 0;
  uint32_t ai = 0, ri = 0;
  while (n_out < b && (ai < n_added || ri < n_row)) {
    gzb_result a;
    if (ai == n_added)
      a = row[ri++];
    else if (ri == n_row || alignment_comp(row[ri], added[ai]) < 0)
      a = added[ai++];
    else
      a = row[ri++];
    if (a.chunk_id != chunk) {  // another chunk's result passes as it is
      out[n_out++] = a;
      continue;
    }
    SubjectStarts *s = nullptr;
    for (int k = 0; k < n_subjects; ++k)
      if (subjects[k].subject == a.subject_id) s = &subjects[k];
    if (!s) {
      s = &subjects[n_subjects++];
      s->subject = a.subject_id;
      s->n = 0;
    }
    if (s->n >= p.max_number_one_subject_results) continue;
    // accepted results of this subject whose listed position lies in
    // [start_d, end_d) must not contain the candidate
    int it = first_not_below(s->starts, 0, s->n, a.start_d);
    const int insert_at = it;
    const int it_end = first_not_below(s->starts, it, s->n, a.end_d);
    bool keep = true;
    for (; it < it_end; ++it)
      if (contained(out[s->starts[it].result], a)) {
        keep = false;
        break;
      }
    if (!keep) continue;
    // the reference lists the new result under its query start
    for (int k = s->n; k > insert_at; --k) s->starts[k] = s->starts[k - 1];
    s->starts[insert_at] = Start{a.start_q, n_out};
    ++s->n;
    out[n_out++] = a;
  }
  for (uint32_t i = 0; i < n_out; ++i) row[i] = out[i];
  return n_out;
}

}  // namespace

extern "C" int gzb_merge_chunk_results(const gzb_params *params, uint32_t number_queries,
                                       const uint32_t *chunk_counts,
                                       const gzb_result *chunk_results, uint32_t *counts,
                                       gzb_result *results) {
  GZB_CHECK(params && (number_queries == 0 ||
                       (chunk_counts && chunk_results && counts && results)),
            GZB_ERR_INVALID, "null argument");
  const gzb_params &p = *params;
  GZB_CHECK(p.max_number_results >= 1 && p.max_number_results <= 32 &&
                p.max_number_one_subject_results >= 1,
            GZB_ERR_INVALID, "max_number_results must be 1..32 and the per-subject limit >= 1");
  const uint32_t b = (uint32_t)p.max_number_results;
  for (uint32_t q = 0; q < number_queries; ++q)
    GZB_CHECK(chunk_counts[q] <= b && counts[q] <= b, GZB_ERR_INVALID,
              "query %u holds more than %u results", q, b);
  for (uint32_t q = 0; q < number_queries; ++q) {
    const gzb_result *c = chunk_results + (size_t)q * b;
    for (uint32_t i = 1; i < chunk_counts[q]; ++i)
      GZB_CHECK(c[i].chunk_id == c[0].chunk_id, GZB_ERR_INVALID,
                "query %u: the added results come from more than one chunk", q);
  }
  gzb_result added[kMaxResults];
  for (uint32_t q = 0; q < number_queries; ++q) {
    if (chunk_counts[q] == 0) continue;  // nothing added: the row stays
    std::copy(chunk_results + (size_t)q * b, chunk_results + (size_t)q * b + chunk_counts[q],
              added);
    counts[q] = merge_row(p, added, chunk_counts[q], results + (size_t)q * b, counts[q]);
  }
  return GZB_OK;
}
