"""Device index cache: a chunk's index exported to host memory and set again
from the blob gives the same index arrays and the same presearch results as
building it; blobs of other parameters or other chunks are refused."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engines():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gzb import native as N
    a, b = N.PresearchEngine(0), N.PresearchEngine(0)
    yield a, b
    a.close()
    b.close()


@pytest.mark.parametrize("clustering", [True, False])
def test_index_roundtrip(engines, clustering):
    a, b = engines
    p = P.make_params(clustering=clustering)
    db = W.make_database(1200, 2401, median=250)
    q = W.make_queries(db, 80, 2402, median=250)
    for e in (a, b):
        e.set_params(p)
    a.set_database(db)
    blob = a.export_index()
    b.set_database(db, index=blob)
    ia, ib = a.index_arrays(), b.index_arrays()
    for name in ia:
        assert np.array_equal(ia[name], ib[name]), name
    for e in (a, b):
        e.set_queries(q)
        e.reset_results()
        e.presearch(0)
    ra, rb = a.results(), b.results()
    assert all(np.array_equal(x, y) for x, y in zip(ra, rb))
    assert sum(len(x) for x in ra) > 0


def test_index_blob_refused_for_other_chunks_and_parameters(engines):
    from gzb import native as N
    a, b = engines
    p = P.make_params()
    db = W.make_database(600, 2501, median=250)
    other = W.make_database(600, 2502, median=250)
    a.set_params(p)
    a.set_database(db)
    blob = a.export_index()
    b.set_params(p)
    with pytest.raises(N.GzbError, match="another chunk"):
        b.set_database(other, index=blob)
    with pytest.raises(N.GzbError, match="truncated"):
        b.set_database(db, index=blob[: len(blob) // 2])
    bad = blob.copy()
    bad[0] ^= 1
    with pytest.raises(N.GzbError, match="not an index blob"):
        b.set_database(db, index=bad)
    b.set_params(P.make_params(clustering=False))
    with pytest.raises(N.GzbError, match="other index parameters"):
        b.set_database(db, index=blob)


def test_reference_index_file_loads(engines, oracle):
    """The reference's .sdp file of a chunk (committed fixture) converted on
    the host is byte for byte the blob the device build exports, and the
    presearch from it matches the oracle."""
    import importlib.util
    import os
    from gzb import native as N
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                        "make_reference_index.py")
    spec = importlib.util.spec_from_file_location("make_reference_index", path)
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    a, b = engines
    p = P.make_params()
    db = g.chunk()
    with open(g.FIXTURE, "rb") as f:
        blob = N.index_blob_from_reference(p, f.read(), db)
    a.set_params(p)
    a.set_database(db)
    assert np.array_equal(a.export_index(), blob)
    b.set_params(p)
    b.set_database(db, index=blob)
    q = W.make_queries(db, 40, 2601, median=80)
    b.set_queries(q)
    b.reset_results()
    b.presearch(0)
    res, _, _ = oracle.presearch(p, db, q)
    got = b.results()
    assert all(np.array_equal(got[i], res[i]) for i in range(q.number))
    assert sum(len(x) for x in got) > 0
