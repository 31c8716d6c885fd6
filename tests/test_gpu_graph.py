"""Graph mode: the presearch captured as one CUDA graph per resident chunk
(and query set) gives the eager path's results and counters, falls back
eagerly when its capacities overflow, and keeps one graph per chunk when
stored chunks are swapped in."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

pytestmark = pytest.mark.gpu

COUNTERS = ("distance_seeds", "ungapped_seeds", "ungapped_hits", "chained_hits",
            "gapped_extensions", "gapped_cells")


@pytest.fixture(scope="module")
def native():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gzb import native as N
    return N


def _eager(N, params, db, q, schedule):
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        e.presearch(schedule)
        return e.results(), e.counters(), e.hits()
    finally:
        e.close()


def _same(a, b):
    assert len(a) == len(b)
    for i, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), i


@pytest.mark.parametrize("clustering", [True, False])
def test_graph_presearch_matches_eager(native, clustering):
    N = native
    params = P.make_params(clustering=clustering)
    db = W.make_database(1500, 901, median=250)
    q = W.make_queries(db, 120, 902, median=250)
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        e.set_graph(True)
        for schedule in (N.SCHEDULE_PLAIN, N.SCHEDULE_BATCHED):
            res, cnt, hits = _eager(N, params, db, q, schedule)
            for _ in range(2):  # captured, then replayed
                e.reset_results()
                e.presearch(schedule)
                _same(e.results(), res)
                got = e.counters()
                for k in COUNTERS:
                    assert got[k] == cnt[k], (schedule, k)
                gh = e.hits()
                assert all(np.array_equal(a, b) for a, b in zip(gh, hits))
        captures, replays, fallbacks = e.graph_stats()
        assert captures == 2 and replays == 4 and fallbacks == 0
    finally:
        e.close()


def test_graph_overflow_falls_back_eagerly(native, params):
    N = native
    db = W.make_database(1500, 903, median=250)
    q = W.make_queries(db, 120, 904, median=250)
    res, cnt, _ = _eager(N, params, db, q, N.SCHEDULE_BATCHED)
    assert cnt["ungapped_hits"] > 100
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        e.set_graph(True)
        e.reserve(100, 100)          # far too small: the graph run overflows
        e.reset_results()
        e.presearch(N.SCHEDULE_BATCHED)
        _same(e.results(), res)      # redone eagerly, merged once
        assert e.graph_stats()[2] == 1
        e.reset_results()
        e.presearch(N.SCHEDULE_BATCHED)  # grown capacities: a graph run
        _same(e.results(), res)
        captures, replays, fallbacks = e.graph_stats()
        assert captures == 2 and replays == 2 and fallbacks == 1
    finally:
        e.close()


def test_one_graph_per_stored_chunk(native, params):
    N = native
    chunks = [W.make_database(800, 910 + k, median=250) for k in range(3)]
    seqs = []
    for k, db in enumerate(chunks):
        seqs += W.query_sequences(W.make_queries(db, 25, 920 + k, median=250))
    q = W.pack_queries(seqs)
    ref = N.PresearchEngine(0)
    try:
        ref.set_params(params)
        ref.set_queries(q)
        ref.reset_results()
        for k, db in enumerate(chunks):
            ref.set_database(db, chunk_id=k)
            ref.presearch(N.SCHEDULE_BATCHED)
        exp = ref.results()
    finally:
        ref.close()
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_queries(q)
        for k, db in enumerate(chunks):
            e.set_database(db, chunk_id=k)
            e.swap_database(k)
        e.set_graph(True)
        for _ in range(3):
            e.reset_results()
            for k in range(len(chunks)):
                e.swap_database(k)
                e.presearch(N.SCHEDULE_BATCHED)
                e.swap_database(k)
            _same(e.results(), exp)
        captures, replays, fallbacks = e.graph_stats()
        assert fallbacks == 0 and replays == 9 and captures == len(chunks)
    finally:
        e.close()


def test_graph_stage_times(native, params):
    """Graph runs report their stage times from device clock stamps."""
    N = native
    db = W.make_database(1500, 905, median=250)
    q = W.make_queries(db, 120, 906, median=250)
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        e.set_graph(True)
        e.presearch(N.SCHEDULE_BATCHED)
        st = e.stage_ms()
        assert all(v >= 0 for v in st.values()), st
        parts = st["lookup"] + st["seed_ungapped"] + st["chain"] + st["gapped"] + st["merge"]
        assert abs(parts - st["total"]) < 1e-3 + 1e-3 * st["total"]
        assert 0 < st["seed_kernels"] <= st["seed_ungapped"] + 1e-3
        assert st["gapped"] > 0
    finally:
        e.close()


@pytest.mark.parametrize("kernel", ["rows", "lane"])
def test_graph_with_cost_model_order(native, params, kernel):
    """The cost-model order inside the graph: same results as the eager
    path, the order coming from the model's predictions on the device."""
    N = native
    db = W.make_database(1500, 907, median=250)
    q = W.make_queries(db, 120, 908, median=250)
    model = N.cost_model_init(seed=5)
    ker = {"rows": N.GAPPED_KERNEL_ROWS, "lane": N.GAPPED_KERNEL_LANE}[kernel]

    def engine(graph):
        e = N.PresearchEngine(0)
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        e.set_cost_model(model)
        e.set_tile(N.SCHEDULE_BATCHED, N.TILE_GAPPED_KERNEL, ker)
        e.set_tile(N.SCHEDULE_BATCHED, N.TILE_ORDER, N.ORDER_MODEL)
        e.set_graph(graph)
        return e

    ref, e = engine(False), engine(True)
    try:
        ref.presearch(N.SCHEDULE_BATCHED)
        exp, cnt = ref.results(), ref.counters()
        for _ in range(2):
            e.reset_results()
            e.presearch(N.SCHEDULE_BATCHED)
            _same(e.results(), exp)
            got = e.counters()
            for k in COUNTERS:
                assert got[k] == cnt[k], k
        captures, replays, fallbacks = e.graph_stats()
        assert captures == 1 and replays == 2 and fallbacks == 0
    finally:
        ref.close()
        e.close()
