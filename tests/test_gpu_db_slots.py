"""Stored and prefetched database chunks: a database of several chunks
searched through the engine's slots (every chunk stored on the device, or
streamed through two slots with copies on a side stream) gives the merged
results of setting each chunk in turn."""
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


def test_stored_chunks_match_sequential(native, params):
    N = native
    chunks, q = _database()
    exp = _sequential(N, params, chunks, q)
    assert sum(len(r) for r in exp) > 0
    assert len({int(x["chunk_id"]) for r in exp for x in r}) == len(chunks)
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


def test_prefetched_chunks_match_sequential(native, params):
    import torch
    N = native
    chunks, q = _database()
    exp = _sequential(N, params, chunks, q)
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


def test_chunk_shards_match_sequential(native, params):
    """Each chunk searched alone (results reset before it), its lists merged
    on the host in chunk order (the exchange step of chunks spread over
    GPUs, here one process), equals one engine searching the chunks in
    turn."""
    from gzb import shards as S
    N = native
    chunks, q = _database()
    exp = _sequential(N, params, chunks, q)
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
