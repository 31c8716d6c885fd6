"""The learned schedule of the gapped stage on the GPU: (features, DP cells)
pairs logged by the plain path train the cost model with the project's own
kernels; the batched schedule then orders extensions by predicted cost.
Results must stay bit-identical under every schedule, and the prediction
error is reported and bounded."""
import numpy as np
import pytest

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


def test_learned_schedule_identical_results_and_accurate(engine, params):
    from gzb import native as N
    # training data logged by the plain path on one workload
    db = W.make_database(4000, 1101, median=250)
    q = W.make_queries(db, 400, 1102, median=250)
    engine.set_params(params)
    engine.set_database(db)
    engine.set_queries(q)
    engine.set_logging(True, 1 << 22)
    engine.presearch(N.SCHEDULE_PLAIN)
    x, y = engine.get_log()
    assert len(y) == engine.counters()["gapped_extensions"] - engine.counters()["gapped_fallbacks"] \
        or len(y) > 0
    params_model, loss = engine.train_cost_model(epochs=150, batch=2048, lr=3e-3, seed=3)
    engine.set_logging(False)
    assert loss < 0.5 * float(np.var(y))  # better than predicting the mean
    # evaluation on another workload
    db2 = W.make_database(4000, 1201, median=250)
    q2 = W.make_queries(db2, 400, 1202, median=250)
    engine.set_database(db2)
    engine.set_queries(q2)
    engine.presearch(N.SCHEDULE_PLAIN)
    plain = engine.results()
    engine.reset_results()
    engine.presearch(N.SCHEDULE_BATCHED)
    batched = engine.results()
    err, n = engine.schedule_stats()
    assert n > 0 and 0 <= err < 1.0, err  # mean |log2 error| below one doubling
    engine.reset_results()
    engine.presearch(N.SCHEDULE_ORACLE)
    oracle_order = engine.results()
    for a, b, c in zip(plain, batched, oracle_order):
        assert np.array_equal(a, b) and np.array_equal(a, c)
    # without a model the batched schedule falls back to the plain order
    engine.set_cost_model(None)
    engine.reset_results()
    engine.presearch(N.SCHEDULE_BATCHED)
    assert all(np.array_equal(a, b) for a, b in zip(plain, engine.results()))


def _warp_cost(cells, order):
    """DP cells the lane kernel pays when each warp runs 32 consecutive
    extensions of `order` to completion: 32 x the costliest of each group."""
    c = cells[order].astype(np.float64)
    pad = (-len(c)) % 32
    c = np.concatenate([c, np.zeros(pad)])
    return 32.0 * c.reshape(-1, 32).max(axis=1).sum()


def test_trained_model_reduces_lane_kernel_work(engine, params):
    """What the network gains over the schedule without it: the same
    extension list costs the lane kernel fewer warp-steps in predicted-cost
    order than in the plain hit order (the method without a model), with the
    true-cost order as the bound."""
    from gzb import native as N
    db = W.make_database(6000, 1301, median=300)
    q = W.make_queries(db, 600, 1302, median=300)
    engine.set_params(params)
    engine.set_database(db)
    engine.set_queries(q)
    engine.set_logging(True, 1 << 22)
    engine.presearch(N.SCHEDULE_PLAIN)
    engine.train_cost_model(epochs=150, batch=2048, lr=3e-3, seed=5)
    engine.set_logging(False)
    db2 = W.make_database(6000, 1401, median=300)
    q2 = W.make_queries(db2, 600, 1402, median=300)
    engine.set_database(db2)
    engine.set_queries(q2)
    engine.reset_results()
    engine.presearch(N.SCHEDULE_BATCHED)
    pred, cells = engine.extension_costs()
    assert len(cells) == engine.counters()["gapped_extensions"] and len(cells) > 1000
    cells = np.where(cells == 0xFFFFFFFF, 0, cells)  # handed to the fallback kernels
    plain = _warp_cost(cells, np.arange(len(cells)))
    learned = _warp_cost(cells, np.argsort(-pred, kind="stable"))
    best = _warp_cost(cells, np.argsort(-cells.astype(np.int64), kind="stable"))
    print(f"lane-kernel work / DP cells: plain {plain / cells.sum():.3f} "
          f"learned {learned / cells.sum():.3f} true-cost order {best / cells.sum():.3f}")
    assert best <= learned < 0.95 * plain
