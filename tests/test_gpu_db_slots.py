"""A database of several chunks, searched chunk after chunk (each set in
turn), through the engine's slots (every chunk stored on the device, or
streamed through two slots with copies on a side stream) and as shards
merged on the host: every mode gives the oracle's chunk loop, i.e. each
chunk's presearch merged into the running lists by AddResults in chunk
order (src/aligner_gpu_presearch_thread.cpp:214-640 with
AlignerCommon::AddResults, src/aligner_common.h:147-274)."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def native():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gzb import native as N
    return N


def _database(n_chunks=3):
    chunks = [W.make_database(900, 800 + k, median=250) for k in range(n_chunks)]
    seqs = []
    for k, db in enumerate(chunks):
        q = W.make_queries(db, 30, 850 + k, median=250)
        seqs += W.query_sequences(q)
    return chunks, W.pack_queries(seqs)


def _oracle_chunk_loop(oracle, params, chunks, q):
    """Each chunk's presearch lists (chunk_id set to the chunk) merged into
    the running lists in chunk order.  Merging a chunk's own top-b lists
    gives the running merge of its raw candidates (tests/test_shards.py
    checks that on the CPU)."""
    import oracle as O
    running = [np.zeros(0, O.RESULT_DTYPE) for _ in range(q.number)]
    for k, db in enumerate(chunks):
        res, _, _ = oracle.presearch(params, db, q)
        for i in range(q.number):
            added = res[i].copy()
            added["chunk_id"] = k
            running[i] = oracle.add_results(params, db, added, running[i])
    return running


@pytest.fixture(scope="module")
def case(oracle, params):
    chunks, q = _database()
    exp = _oracle_chunk_loop(oracle, params, chunks, q)
    assert sum(len(r) for r in exp) > 0
    assert len({int(x["chunk_id"]) for r in exp for x in r}) == len(chunks)
    return chunks, q, exp


def _sequential(N, params, chunks, q):
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_queries(q)
        e.reset_results()
        for k, db in enumerate(chunks):
            e.set_database(db, chunk_id=k)
            e.presearch(N.SCHEDULE_BATCHED)
        return e.results()
    finally:
        e.close()


def _same(a, b):
    assert len(a) == len(b)
    for i, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), i


def test_sequential_chunks_match_oracle(native, params, case):
    chunks, q, exp = case
    _same(_sequential(native, params, chunks, q), exp)


def test_stored_chunks_match_oracle(native, params, case):
    N = native
    chunks, q, exp = case
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_queries(q)
        for k, db in enumerate(chunks):
            e.set_database(db, chunk_id=k)   # index built on the device
            e.swap_database(k)               # stored compactly in slot k
        for rounds in range(2):              # the stored chunks stay valid
            e.reset_results()
            for k in range(len(chunks)):
                e.swap_database(k)
                e.presearch(N.SCHEDULE_BATCHED)
                e.swap_database(k)
            _same(e.results(), exp)
    finally:
        e.close()


def test_prefetched_chunks_match_oracle(native, params, case):
    import torch
    N = native
    chunks, q, exp = case
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        blobs = []
        for db in chunks:
            e.set_database(db)
            blobs.append(e.export_index())
        e.set_queries(q)
        e.reset_results()
        side = torch.cuda.Stream()
        e.prefetch_database(0, chunks[0], blobs[0], chunk_id=0, stream=side)
        e.swap_database(0)
        for k in range(len(chunks)):
            if k + 1 < len(chunks):  # the next chunk's copies overlap this search
                e.prefetch_database(1, chunks[k + 1], blobs[k + 1], chunk_id=k + 1,
                                    stream=side)
            e.presearch(N.SCHEDULE_BATCHED)
            if k + 1 < len(chunks):
                e.swap_database(1)
        _same(e.results(), exp)
    finally:
        e.close()


def test_slot_refusals(native, params):
    N = native
    chunks, q = _database(2)
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(chunks[0])
        blob0 = e.export_index()
        with pytest.raises(N.GzbError):
            e.swap_database(64)
        with pytest.raises(N.GzbError):   # another chunk's index
            e.prefetch_database(0, chunks[1], blob0)
        bad = W.Database(codes=chunks[0].codes.copy(), offsets=chunks[0].offsets,
                         number_sequences=chunks[0].number_sequences)
        # a residue code out of range keeps its chunk out (the index check
        # covers the offsets and both ends, so alter the middle)
        bad.codes[len(bad.codes) // 2] = 40
        e.prefetch_database(0, bad, blob0)
        with pytest.raises(N.GzbError, match="below 32"):
            e.swap_database(0)
        # the resident chunk is untouched and still searches
        e.set_queries(q)
        e.presearch(N.SCHEDULE_PLAIN)
    finally:
        e.close()


def test_chunk_shards_match_oracle(native, params, case):
    """Each chunk searched alone (results reset before it), its lists merged
    on the host in chunk order (the exchange step of chunks spread over
    GPUs, here one process), equals the oracle's chunk loop."""
    from gzb import shards as S
    N = native
    chunks, q, exp = case
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_queries(q)
        counts, records = S.ChunkShards().search(e, params, chunks, N.SCHEDULE_BATCHED)
    finally:
        e.close()
    b = int(params["max_number_results"])
    rows = records.reshape(q.number, b)
    _same([rows[i, :counts[i]] for i in range(q.number)], exp)
