"""Six-frame translation on the GPU (query preparation of translated-DNA
searches) against the oracle's restatement of TranslatedDnaQuery, and the
presearch of translated queries against the oracle, bit for bit."""
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


def _reads(rng, lengths):
    # mostly ACGT with some N, lowercase and other IUPAC letters
    letters = np.frombuffer(b"ACGTACGTACGTACGTacgtNNRYKM", np.uint8)
    seqs = [letters[rng.integers(0, len(letters), int(n))] for n in lengths]
    offsets = np.zeros(len(seqs) + 1, np.uint64)
    offsets[1:] = np.cumsum([len(s) for s in seqs])
    dna = np.concatenate(seqs) if seqs else np.zeros(0, np.uint8)
    return dna, offsets


def _check(native, oracle, dna, offsets):
    codes, offs, lens = native.translate_reads(dna, offsets, P.DELIMITER)
    n = len(offsets) - 1
    assert len(offs) == n and len(lens) == n
    for r in range(n):
        read = dna[int(offsets[r]):int(offsets[r + 1])].tobytes()
        exp = oracle.translate_query(read, P.DELIMITER)
        got = codes[int(offs[r]):int(offs[r]) + int(lens[r])]
        assert np.array_equal(got, exp), (r, len(read))
    if n:
        assert len(codes) == int(offs[-1]) + int(lens[-1])


def test_translation_matches_oracle(native, oracle):
    rng = np.random.default_rng(40)
    lengths = list(range(0, 40)) + list(rng.integers(3, 3000, 300)) + [150] * 200
    rng.shuffle(lengths)
    dna, offsets = _reads(rng, lengths)
    _check(native, oracle, dna, offsets)


def test_translation_edges(native, oracle):
    rng = np.random.default_rng(41)
    # one read, only short reads, and one long read
    for lengths in ([150], [0, 1, 2, 0], [1, 2, 3, 4, 5], [100000]):
        dna, offsets = _reads(rng, lengths)
        _check(native, oracle, dna, offsets)
    codes, offs, lens = native.translate_reads(np.zeros(0, np.uint8), np.zeros(1, np.uint64),
                                               P.DELIMITER)
    assert len(codes) == 0 and len(offs) == 0


def test_translated_presearch_matches_oracle(native, oracle, params):
    db = W.make_database(1500, 701, median=250)
    reads = W.make_reads(db, 160, 702)
    codes, offs, lens = native.translate_reads(reads.dna, reads.offsets, P.DELIMITER)
    q = W.translated_queries(codes, offs, lens, sources=reads.sources)
    e = native.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        res, cnt, hits = oracle.presearch(params, db, q)
        assert cnt["gapped_extensions"] > 0
        for schedule in (native.SCHEDULE_PLAIN, native.SCHEDULE_BATCHED):
            e.reset_results()
            e.presearch(schedule)
            got = e.results()
            gc = e.counters()
            for k in ("distance_seeds", "ungapped_seeds", "ungapped_hits", "chained_hits",
                      "gapped_extensions", "gapped_cells"):
                assert gc[k] == cnt[k], (schedule, k, gc[k], cnt[k])
            for i in range(q.number):
                assert np.array_equal(got[i], res[i]), (schedule, i)
        # planted fragments find their source protein
        found = sum(1 for i in range(q.number) if reads.sources[i] >= 0 and
                    any(int(r["subject_id"]) == int(reads.sources[i]) for r in got[i]))
        assert found >= 0.5 * int((reads.sources >= 0).sum())
    finally:
        e.close()
