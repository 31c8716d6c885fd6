"""Database chunks spread over ranks: each chunk's own top-b lists, merged
in chunk order by gzb_merge_chunk_results (host), equal the running
AddResults merge of every chunk's raw candidates (the oracle's restatement
of src/aligner_common.h:147-274), ties and containment included; two gloo
ranks exchanging their chunks' lists reach the same lists."""
import os
import socket

import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

N_CHUNKS = 5
N_QUERIES = 40


def _params():
    # several results per subject, so containment decides as well as the limit
    p = P.make_params(max_number_results=10)
    p["max_number_one_subject_results"] = 8
    return p


def _chunks():
    # chunks with the same residues (and so the same positions), so that
    # candidates of different chunks tie exactly and chunk order decides
    db = W.make_database(30, 900, median=60)
    return [db] * N_CHUNKS


def _raw(db, chunk, query):
    """Candidates of one query in one chunk: some shared by every chunk
    (exact ties across chunks), the others the chunk's own; narrow scores
    (ties), copies with the same start or end (contained) and exact ties of
    the ordering that are not contained."""
    return np.concatenate([_candidates(db, chunk, np.random.default_rng(query), 8),
                           _candidates(db, chunk, np.random.default_rng(10_000 * chunk + query),
                                       None)])


def _candidates(db, chunk, rng, n):
    from gzb import native as N
    if n is None:
        n = int(rng.integers(0, 30))
    r = np.zeros(n, N.RESULT_DTYPE)
    if n == 0:
        return r
    subj = rng.integers(0, db.number_sequences, n)
    first = db.offsets[subj].astype(np.int64)
    last = db.offsets[subj + 1].astype(np.int64) - 2  # before the delimiter
    sd = first + (rng.random(n) * (last - first) / 2).astype(np.int64)
    ed = np.minimum(sd + rng.integers(0, 20, n), last)
    sq = rng.integers(1, 300, n)
    eq = sq + (ed - sd) + rng.integers(0, 3, n)
    r["chunk_id"] = chunk
    r["subject_id"] = -1
    r["score"] = rng.integers(20, 26, n)
    r["start_d"], r["end_d"], r["start_q"], r["end_q"] = sd, ed, sq, eq
    r["hit_q"], r["hit_d"] = sq, sd
    k = n // 3
    if k:
        same_start = r[:k].copy()
        same_start["end_q"] = same_start["start_q"] + (same_start["end_q"] - same_start["start_q"]) // 2
        same_start["end_d"] = same_start["start_d"] + (same_start["end_d"] - same_start["start_d"]) // 2
        tied = r[:k].copy()
        tied["start_q"] += 1
        tied["end_q"] += 1
        r = np.concatenate([r, same_start, tied])
    return r[rng.permutation(len(r))]


def _rows(params, lists):
    """Per-query lists -> (counts, records) in the ABI's layout."""
    from gzb import native as N
    b = int(params["max_number_results"])
    counts = np.array([len(x) for x in lists], np.uint32)
    records = np.zeros(len(lists) * b, N.RESULT_DTYPE)
    for i, x in enumerate(lists):
        records[i * b:i * b + len(x)] = x
    return counts, records


def _chunk_lists(oracle, params, chunks, which):
    """Each listed chunk's own lists: AddResults of its candidates into
    empty lists (what the engine holds after a reset and that chunk)."""
    return {c: _rows(params, [oracle.add_results(params, chunks[c], _raw(chunks[c], c, q), [])
                              for q in range(N_QUERIES)])
            for c in which}


def _expected(oracle, params, chunks):
    """The running merge: every chunk's raw candidates added in turn."""
    from gzb import native as N
    out = []
    for q in range(N_QUERIES):
        res = np.zeros(0, N.RESULT_DTYPE)
        for c, db in enumerate(chunks):
            res = oracle.add_results(params, db, _raw(db, c, q), res)
        out.append(res)
    return _rows(params, out)


def _same(a, b):
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.int32), b[1].view(np.int32))


def test_chunk_lists_merged_in_order_equal_the_running_merge(oracle):
    from gzb import shards as S
    params = _params()
    chunks = _chunks()
    local = _chunk_lists(oracle, params, chunks, range(N_CHUNKS))
    exp = _expected(oracle, params, chunks)
    assert exp[0].sum() > N_QUERIES  # non-trivial lists
    assert len({int(x) for x in exp[1]["chunk_id"][:int(exp[0].sum())]}) > 1
    got = S.merge_in_order(params, [local[c] for c in range(N_CHUNKS)])
    _same(got, exp)
    # the chunks tie exactly, so the order of the merge matters
    rev = S.merge_in_order(params, [local[c] for c in reversed(range(N_CHUNKS))])
    assert not np.array_equal(rev[1].view(np.int32), exp[1].view(np.int32))
    # one process holding every chunk: the exchange is the identity
    sh = S.ChunkShards()
    _same(sh.merged(params, sh.exchange(params, N_CHUNKS, N_QUERIES, local)), exp)
    # query slices merge independently
    b = int(params["max_number_results"])
    part = S.merge_in_order(params, [local[c] for c in range(N_CHUNKS)], 7, 23)
    assert np.array_equal(part[0], exp[0][7:23])
    assert np.array_equal(part[1].view(np.int32), exp[1][7 * b:23 * b].view(np.int32))


def test_merge_of_raw_candidates_is_add_results(oracle):
    """Raw candidates crowded into a few subjects (up to 32 kept per
    subject, so the per-subject start lists grow long and, keyed by query
    start but placed by database start, unsorted) merged into empty lists
    give the oracle's AddResults exactly."""
    from gzb import native as N
    params = P.make_params(max_number_results=32)
    params["max_number_one_subject_results"] = 32
    db = W.make_database(3, 77, median=400)
    b = 32
    n_cases = 300
    counts = np.zeros(n_cases, np.uint32)
    records = np.zeros(n_cases * b, N.RESULT_DTYPE)
    added_counts = np.zeros(n_cases, np.uint32)
    added = np.zeros(n_cases * b, N.RESULT_DTYPE)
    expected = []
    for case in range(n_cases):
        rng = np.random.default_rng(5000 + case)
        n = int(rng.integers(1, b + 1))
        subj = rng.integers(0, db.number_sequences, n)
        first = db.offsets[subj].astype(np.int64)
        sd = first + rng.integers(0, 60, n)
        ed = sd + rng.integers(0, 40, n)
        sq = rng.integers(0, 120, n)  # query starts unrelated to database starts
        r = np.zeros(n, N.RESULT_DTYPE)
        r["chunk_id"] = 3
        r["subject_id"] = subj
        r["score"] = rng.integers(30, 33, n)
        r["start_d"], r["end_d"], r["start_q"] = sd, ed, sq
        r["end_q"] = sq + (ed - sd)
        added_counts[case] = n
        added[case * b:case * b + n] = r
        expected.append(oracle.add_results(params, db, r, []))
    N.merge_chunk_results(params, added_counts, added, counts, records)
    exp = _rows(params, expected)
    _same((counts, records), exp)
    assert exp[0].min() < exp[0].max()  # containment rejected some, not all


def test_merge_refuses_rows_over_capacity_and_mixed_chunks(oracle):
    from gzb import native as N
    params = _params()
    b = int(params["max_number_results"])
    counts = np.zeros(2, np.uint32)
    records = np.zeros(2 * b, N.RESULT_DTYPE)
    over = np.array([b + 1, 0], np.uint32)
    with pytest.raises(N.GzbError):
        N.merge_chunk_results(params, over, np.zeros(2 * b, N.RESULT_DTYPE), counts, records)
    mixed = np.zeros(2 * b, N.RESULT_DTYPE)
    mixed["chunk_id"][:2] = [0, 1]
    with pytest.raises(N.GzbError, match="more than one chunk"):
        N.merge_chunk_results(params, np.array([2, 0], np.uint32), mixed, counts, records)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from datetime import timedelta

    import oracle as O
    import torch.distributed as dist
    from gzb import shards as S
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        params = _params()
        chunks = _chunks()
        sh = S.ChunkShards(dist, "cpu")
        mine = S.chunks_of(rank, world, N_CHUNKS)
        local = _chunk_lists(O.Oracle(), params, chunks, mine)
        merged = sh.merged(params, sh.exchange(params, N_CHUNKS, N_QUERIES, local))
        out.put((rank, mine, merged[0], merged[1].view(np.int32)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_their_chunks(oracle):
    pytest.importorskip("torch")
    import torch.multiprocessing as mp
    params = _params()
    exp = _expected(oracle, params, _chunks())
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(m for _, m, _, _ in got) == [[0, 2, 4], [1, 3]]
    for _, _, counts, words in got:
        assert np.array_equal(counts, exp[0])
        assert np.array_equal(words, exp[1].view(np.int32))


class _FakeEngine:
    """The engine calls ChunkShards.search makes, answered on the host: a
    chunk's lists are its candidates added into empty lists (what the
    engine holds after a reset and one presearch of that chunk)."""

    def __init__(self, oracle, params):
        self.oracle, self.params = oracle, params
        self.number_queries = N_QUERIES
        self.calls = []

    def set_database(self, db, chunk_id=0):
        self.db, self.chunk = db, chunk_id
        self.calls.append(("set_database", chunk_id))

    def reset_results(self):
        self.calls.append(("reset_results",))

    def presearch(self, schedule):
        self.calls.append(("presearch", schedule))
        self.rows = _rows(self.params, [
            self.oracle.add_results(self.params, self.db, _raw(self.db, self.chunk, q), [])
            for q in range(N_QUERIES)])

    def result_rows(self):
        return self.rows


def test_search_drives_the_engine_chunk_by_chunk(oracle):
    from gzb import shards as S
    params = _params()
    chunks = _chunks()
    e = _FakeEngine(oracle, params)
    got = S.ChunkShards().search(e, params, chunks, schedule=1)
    _same(got, _expected(oracle, params, chunks))
    assert e.calls == [c for k in range(N_CHUNKS)
                       for c in (("set_database", k), ("reset_results",), ("presearch", 1))]


def test_query_split_covers_every_query_once():
    from gzb import shards as S
    from gzb import workload as W
    db = W.make_database(200, 41, median=120)
    q = W.make_queries(db, 37, 42, median=120)
    for world in (1, 2, 3, 8, 40):
        seen = []
        for r in range(world):
            b, e = S.query_range(r, world, q.number)
            part = S.slice_queries(q, b, e)
            assert part.number == e - b
            for i in range(part.number):
                o, n = int(part.offsets[i]), int(part.lengths[i])
                oo, nn = int(q.offsets[b + i]), int(q.lengths[b + i])
                assert np.array_equal(part.codes[o:o + n], q.codes[oo:oo + nn])
                assert part.cutoffs[i] == q.cutoffs[b + i]
            seen += list(range(b, e))
        assert seen == list(range(q.number))
