"""The build results step on the GPU (AlignerBuildResultsThread::Run,
src/aligner_build_results_thread.h:64-190): both gapped extensions of every
merged result are redone with their edit path, and the alignment length,
mismatches, gap openings and gap extensions must equal the oracle's
restatement of GappedExtender::ExtendOneSide + AlignerCommon::BuildResult,
which is pinned to the reference's own units in test_oracle_pin.py."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

pytestmark = pytest.mark.gpu

FIELDS = ("alignment_length", "mismatches", "gap_openings", "gap_extensions")


@pytest.fixture(scope="module")
def engine():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gzb import native as N
    e = N.PresearchEngine(0)
    yield e
    e.close()


def _check(engine, oracle, params, db, q):
    got = engine.build_alignments()
    res = engine.results()
    n = 0
    for qi in range(q.number):
        assert len(got[qi]) == len(res[qi])
        off = int(q.offsets[qi])
        for a, r in zip(got[qi], res[qi]):
            for k in ("hit_q", "hit_d"):
                assert a[k] == r[k], (qi, k)
            assert a["presearch_score"] == r["score"]
            # the build step's wider X-drop reaches at least the presearch's
            assert a["score"] >= r["score"]
            o = oracle.build_alignment(params, q.codes, off + int(a["hit_q"]), db.codes,
                                       int(a["hit_d"]))
            assert o["score"] == a["score"]
            assert (o["start_q"] - off, o["start_d"], o["end_q"] - off, o["end_d"]) == \
                (a["start_q"], a["start_d"], a["end_q"], a["end_d"])
            for k in FIELDS:
                assert o[k] == a[k], (qi, k, o[k], a[k])
            n += 1
    return n


def test_build_alignments_match_oracle(engine, oracle, params):
    db = W.make_database(1500, 2101, median=250)
    q = W.make_queries(db, 120, 2102, median=250)
    engine.set_params(params)
    engine.set_database(db)
    engine.set_queries(q)
    engine.presearch(0)
    assert _check(engine, oracle, params, db, q) > 50


def test_build_alignments_long_homologs_and_x_drops(engine, oracle):
    # long, gapped homologs and several X-drops, both extension directions
    rng = np.random.default_rng(2201)
    db = W.make_database(300, 2202, median=1200)
    seqs = []
    for s in range(0, 40, 2):
        src = db.codes[db.offsets[s]:db.offsets[s + 1] - 1]
        seqs.append(W.mutate(rng, src, rng.uniform(0.35, 0.9), indel_p=0.05))
    q = W.pack_queries(seqs)
    # (presearch X-drop, build step X-drop): equal, the defaults' ratio, wide
    for cutoff, result_cutoff in ((15, 15), (26, 52), (60, 120)):
        p = P.make_params()
        p["gapped_cutoff"] = cutoff
        p["result_gapped_cutoff"] = result_cutoff
        engine.set_params(p)
        engine.set_database(db)
        engine.set_queries(q)
        engine.presearch(0)
        assert _check(engine, oracle, p, db, q) > 10


def test_build_alignments_skip_other_chunks(engine, oracle, params):
    db0 = W.make_database(800, 2301, median=250)
    db1 = W.make_database(800, 2302, median=250)
    q = W.make_queries(db0, 60, 2303, median=250)
    engine.set_params(params)
    engine.set_queries(q)
    engine.set_database(db0, chunk_id=0)
    engine.presearch(0)
    engine.set_database(db1, chunk_id=1)
    engine.presearch(0)
    got = engine.build_alignments()
    seen = {0: 0, 1: 0}
    for qi in range(q.number):
        for a in got[qi]:
            seen[int(a["chunk_id"])] += 1
            if a["chunk_id"] == 0:
                assert a["alignment_length"] == 0
            else:
                o = oracle.build_alignment(params, q.codes, int(q.offsets[qi]) + int(a["hit_q"]),
                                           db1.codes, int(a["hit_d"]))
                assert all(o[k] == a[k] for k in FIELDS)
    assert seen[0] > 0 and seen[1] > 0
