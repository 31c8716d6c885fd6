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
#include <vector>

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

struct Start {
  uint32_t position, result;  // the reference keys the list by this position
};

struct SubjectStarts {
  int32_t subject;
  std::vector<Start> starts;  // ordered by position
};

size_t first_not_below(const std::vector<Start> &v, size_t from, uint32_t position) {
  return std::lower_bound(v.begin() + from, v.end(), position,
                          [](const Start &s, uint32_t p) { return s.position < p; }) -
         v.begin();
}

// One query: `added` (n_added records of one chunk) merged into `row`
// (n_row records), at most b kept; returns the new count.
uint32_t merge_row(const gzb_params &p, std::vector<gzb_result> &added, gzb_result *row,
                   uint32_t n_row, std::vector<gzb_result> &out) {
  const size_t b = (size_t)p.max_number_results;
  // stable, best first (stable_sort with PresearchedResultGreaterScore)
  std::stable_sort(added.begin(), added.end(), [](const gzb_result &x, const gzb_result &y) {
    return alignment_comp(x, y) > 0;
  });
  const int32_t chunk = added.empty() ? -1 : added[0].chunk_id;
  out.clear();
  std::vector<SubjectStarts> subjects;
  size_t ai = 0, ri = 0;
  while (out.size() < b && (ai < added.size() || ri < n_row)) {
    gzb_result a;
    if (ai == added.size())
      a = row[ri++];
    else if (ri == n_row || alignment_comp(row[ri], added[ai]) < 0)
      a = added[ai++];
    else
      a = row[ri++];
    if (a.chunk_id != chunk) {  // another chunk's result passes as it is
      out.push_back(a);
      continue;
    }
    SubjectStarts *s = nullptr;
    for (auto &x : subjects)
      if (x.subject == a.subject_id) s = &x;
    if (!s) {
      subjects.push_back(SubjectStarts{a.subject_id, {}});
      s = &subjects.back();
    }
    if (s->starts.size() >= (size_t)p.max_number_one_subject_results) continue;
    // accepted results of this subject whose listed position lies in
    // [start_d, end_d) must not contain the candidate
    size_t it = first_not_below(s->starts, 0, a.start_d);
    const size_t insert_at = it;
    const size_t it_end = first_not_below(s->starts, it, a.end_d);
    bool keep = true;
    for (; it < it_end; ++it)
      if (contained(out[s->starts[it].result], a)) {
        keep = false;
        break;
      }
    if (!keep) continue;
    // the reference lists the new result under its query start
    s->starts.insert(s->starts.begin() + insert_at, Start{a.start_q, (uint32_t)out.size()});
    out.push_back(a);
  }
  std::copy(out.begin(), out.end(), row);
  return (uint32_t)out.size();
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
  std::vector<gzb_result> added, out;
  added.reserve(b);
  out.reserve(b);
  for (uint32_t q = 0; q < number_queries; ++q) {
    const gzb_result *c = chunk_results + (size_t)q * b;
    if (chunk_counts[q] == 0) continue;  // nothing added: the row stays
    for (uint32_t i = 1; i < chunk_counts[q]; ++i)
      GZB_CHECK(c[i].chunk_id == c[0].chunk_id, GZB_ERR_INVALID,
                "query %u: the added results come from more than one chunk", q);
    added.assign(c, c + chunk_counts[q]);
    counts[q] = merge_row(p, added, results + (size_t)q * b, counts[q], out);
  }
  return GZB_OK;
}
