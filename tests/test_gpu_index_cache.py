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
