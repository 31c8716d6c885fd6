"""Whole-presearch parity on the GPU: device index, seed survivors and the
per-query top-b lists of the engine against the CPU oracle, bit for bit."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gzb import native as N
    e = N.PresearchEngine(0)
    yield e
    e.close()


def _small(seed_db=501, seed_q=502, n_db=1500, n_q=120, median=250):
    db = W.make_database(n_db, seed_db, median=median)
    q = W.make_queries(db, n_q, seed_q, median=median)
    return db, q


def test_device_index_matches_oracle(engine, oracle, params):
    db, _ = _small()
    engine.set_params(params)
    engine.set_database(db)
    got = engine.index_arrays()
    exp = oracle.db_index(params, db.codes)
    for name in ("nc_keys", "nc_offsets", "nc_values", "rep_keys", "rep_offsets",
                 "rep_positions", "member_offsets", "member_positions"):
        assert np.array_equal(got[name], exp[name]), name


def _compare(engine, oracle, params, db, q, schedule=0):
    engine.set_params(params)
    engine.set_database(db)
    engine.set_queries(q)
    # query hash lists (SeedSearcherGpuQueryParameters) and the device index
    gl = engine.list_arrays()
    el = oracle.query_lists(params, q)
    for name in ("hashes", "offsets", "check_counts", "query_ids", "positions"):
        assert np.array_equal(gl[name], el[name]), name
    gi = engine.index_arrays()
    ei = oracle.db_index(params, db.codes)
    for name in ("nc_keys", "nc_offsets", "nc_values", "rep_keys", "rep_offsets",
                 "rep_positions", "member_offsets", "member_positions"):
        assert np.array_equal(gi[name], ei[name]), name
    engine.presearch(schedule)
    got = engine.results()
    res, cnt, hits = oracle.presearch(params, db, q)
    gh = engine.hits()
    assert np.array_equal(gh[0], hits[0]) and np.array_equal(gh[1], hits[1]) and \
        np.array_equal(gh[2], hits[2]), "ungapped survivors differ"
    gc = engine.counters()
    for k in ("distance_seeds", "ungapped_seeds", "ungapped_hits", "chained_hits",
              "gapped_extensions", "gapped_cells"):
        assert gc[k] == cnt[k], (k, gc[k], cnt[k])
    for i in range(q.number):
        assert np.array_equal(got[i], res[i]), i
    return cnt


def test_presearch_matches_oracle_small(engine, oracle, params):
    db, q = _small()
    cnt = _compare(engine, oracle, params, db, q)
    assert cnt["chained_hits"] > 0 and cnt["gapped_cells"] > 0


def test_presearch_long_queries(engine, oracle, params):
    """Queries longer than the chain filter's shared-memory slots (4,096
    diagonals) keep their slots in global memory; results equal the
    oracle's."""
    db = W.make_database(300, 1201, median=5000, lo=4200, hi=7000)
    q = W.make_queries(db, 24, 1202, median=5000, lo=4200, hi=7000)
    assert int(q.lengths.max()) > 4096
    cnt = _compare(engine, oracle, params, db, q)
    assert cnt["chained_hits"] > 0


def test_presearch_without_clustering(engine, oracle):
    p = P.make_params(clustering=False)
    db, q = _small(601, 602, n_db=800, n_q=60)
    _compare(engine, oracle, p, db, q)


def test_presearch_v2_results(engine, oracle):
    p = P.make_params(max_number_one_subject_results=3, max_number_results=5)
    db, q = _small(701, 702, n_db=800, n_q=60)
    _compare(engine, oracle, p, db, q)


def test_presearch_edge_queries(engine, oracle, params):
    # very short queries (no seeds), a query made of X, and a long homolog
    db = W.make_database(400, 801, median=200)
    rng = np.random.default_rng(9)
    src = db.codes[db.offsets[3]:db.offsets[4] - 1]
    seqs = [W.random_residues(rng, 5), np.full(40, 24, np.uint8), src.copy(),
            W.mutate(rng, src, 0.7), W.random_residues(rng, 9)]
    q = W.pack_queries(seqs)
    _compare(engine, oracle, params, db, q)


def test_presearch_repeated_calls_identical(engine, params):
    db, q = _small(901, 902, n_db=600, n_q=50)
    engine.set_params(params)
    engine.set_database(db)
    engine.set_queries(q)
    engine.presearch(0)
    a = engine.results()
    engine.reset_results()
    engine.presearch(0)
    b = engine.results()
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("kernel,threshold", [(0, 1), (0, 32), (1, 8), (2, 1), (2, 8), (2, 32), (3, 8), (4, 8),
                                              (5, 8), (6, 8), (7, 8), (8, 8)])
def test_presearch_every_gapped_tile(engine, oracle, params, kernel, threshold):
    # every one-thread-per-extension kernel on the work-queue schedule (no
    # model: hit order), and the flat kernel's extreme bookkeeping
    # thresholds, give the oracle's results
    from gzb import native as N
    engine.set_cost_model(None)
    engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_GAPPED_KERNEL, kernel)
    engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_BOOK_THRESHOLD, threshold)
    try:
        db, q = _small(1001, 1002, n_db=800, n_q=60)
        _compare(engine, oracle, params, db, q, schedule=N.SCHEDULE_BATCHED)
    finally:
        engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_GAPPED_KERNEL, -1)
        engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_BOOK_THRESHOLD, -1)


@pytest.mark.parametrize("band,graph", [(32, False), (32, True), (128, False), (128, True)])
def test_presearch_every_band_width(engine, oracle, params, band, graph):
    """The rows kernel with 32 and 128 band columns per lane (a narrower
    band hands more extensions to the warp kernel) gives the oracle's
    results, eager and in graph mode, with the DP's cell count unchanged."""
    from gzb import native as N
    engine.set_cost_model(None)
    engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_GAPPED_KERNEL, N.GAPPED_KERNEL_ROWS)
    engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_BAND_WIDTH, band)
    engine.set_graph(graph)
    try:
        db, q = _small(1101, 1102, n_db=900, n_q=70, median=400)
        cnt = _compare(engine, oracle, params, db, q, schedule=N.SCHEDULE_BATCHED)
        assert cnt["gapped_cells"] > 0
    finally:
        engine.set_graph(False)
        engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_GAPPED_KERNEL, -1)
        engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_BAND_WIDTH, -1)


@pytest.mark.parametrize("graph", [False, True])
def test_dealt_seed_walker_matches_oracle(engine, oracle, params, graph):
    """The dealt seed walker (GZB_SEED_WALKER_DEALT) gives the oracle's
    survivors, counters and lists, eager and in graph mode, and the same
    residue-pair count as the per-unit walker."""
    from gzb import native as N
    db, q = _small(seed_db=701, seed_q=702)
    engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_SEED_WALKER, N.SEED_WALKER_DEALT)
    engine.set_graph(graph)
    try:
        cnt = _compare(engine, oracle, params, db, q, schedule=N.SCHEDULE_BATCHED)
        assert cnt["ungapped_hits"] > 0
        steps = engine.counters()["ungapped_steps"]
        engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_SEED_WALKER, N.SEED_WALKER_UNIT)
        engine.reset_results()
        engine.presearch(N.SCHEDULE_BATCHED)
        assert engine.counters()["ungapped_steps"] == steps
    finally:
        engine.set_graph(False)
        engine.set_tile(N.SCHEDULE_BATCHED, N.TILE_SEED_WALKER, -1)
