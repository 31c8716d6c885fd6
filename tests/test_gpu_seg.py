"""SEG masking and whole query preparation on the GPU against the oracle's
restatement of the reference's SEG filter, translated queries and protein
queries, bit for bit."""
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


def _low_complexity_protein(rng, n):
    letters = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", np.uint8)
    s = letters[rng.integers(0, 20, n)].copy()
    for _ in range(int(rng.integers(0, 5))):
        if n < 2:
            break
        a = int(rng.integers(0, n - 1))
        b = min(n, a + int(rng.integers(5, 80)))
        pool = letters[rng.choice(20, size=int(rng.integers(1, 5)), replace=False)]
        s[a:b] = pool[rng.integers(0, len(pool), b - a)]
    extra = rng.random(n)
    s[extra < 0.02] = ord("*")
    s[(extra >= 0.02) & (extra < 0.03)] = ord("X")
    low = (extra >= 0.03) & (extra < 0.035)
    s[low] = s[low] | 0x20
    s[s == (ord("*") | 0x20)] = ord("*")
    return bytes(s)


def _reads(rng, n_reads):
    out = []
    for _ in range(n_reads):
        n = int(rng.choice([0, 2, 3, 20, 35, 36, 37, 150, 150, 150, int(rng.integers(3, 1200))]))
        if rng.random() < 0.3:  # short tandem repeats translate to low complexity
            unit = bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(rng.integers(1, 7)))])
            out.append((unit * (n // max(len(unit), 1) + 1))[:n])
        else:
            out.append(bytes(np.frombuffer(b"ACGTACGTACGTNacgt", np.uint8)[
                rng.integers(0, 17, n)]))
    offsets = np.zeros(len(out) + 1, np.uint64)
    offsets[1:] = np.cumsum([len(r) for r in out])
    return out, np.frombuffer(b"".join(out), np.uint8).copy(), offsets


def test_translated_queries_with_seg_match_oracle(native, oracle, params):
    rng = np.random.default_rng(70)
    reads, dna, offsets = _reads(rng, 600)
    codes, offs, lens, cut, trig = native.prepare_translated_queries(dna, offsets)
    masked = 0
    for r, read in enumerate(reads):
        exp = oracle.translate_query_seg(read, P.DELIMITER)
        got = codes[int(offs[r]):int(offs[r]) + int(lens[r])]
        assert np.array_equal(got, exp), (r, len(read), read)
        _, _, _, c, t = oracle.query_karlin(params, exp)
        assert (int(cut[r]), int(trig[r])) == (c, t), r
        masked += len(read) >= 36 and bool((got == 24).any())
    assert masked > 20


def test_translated_queries_without_filter(native, oracle, params):
    rng = np.random.default_rng(71)
    reads, dna, offsets = _reads(rng, 200)
    codes, offs, lens, cut, trig = native.prepare_translated_queries(dna, offsets, filter=False)
    for r, read in enumerate(reads):
        exp = oracle.translate_query(read, P.DELIMITER)
        assert np.array_equal(codes[int(offs[r]):int(offs[r]) + int(lens[r])], exp), r
        _, _, _, c, t = oracle.query_karlin(params, exp)
        assert (int(cut[r]), int(trig[r])) == (c, t), r


def test_protein_queries_with_seg_match_oracle(native, oracle, params):
    rng = np.random.default_rng(72)
    prots = [_low_complexity_protein(rng, int(rng.choice(
        [0, 1, 5, 11, 12, 13, 50, int(rng.integers(12, 800)), int(rng.integers(800, 5000))])))
        for _ in range(500)]
    seqs = [native.encode_protein_for_seg(p) for p in prots]
    q = W.pack_queries(seqs, cutoffs=(np.zeros(len(seqs), np.int32),
                                      np.zeros(len(seqs), np.int32)))
    codes, cut, trig = native.prepare_protein_queries(q.codes, q.offsets, q.lengths)
    masked = 0
    for i, p in enumerate(prots):
        exp = oracle.protein_query_seg(p, P.DELIMITER)
        o, n = int(q.offsets[i]), int(q.lengths[i])
        # the held buffer's last code is dropped when queries are concatenated
        assert np.array_equal(codes[o:o + n - 1], exp[:-1]), (i, len(p), p)
        _, _, _, c, t = oracle.query_karlin(params, exp)
        assert (int(cut[i]), int(trig[i])) == (c, t), (i, len(p))
        masked += bool((codes[o + 1:o + n - 1] == 24).any())
    assert masked > 100


def test_seg_prepared_queries_search_like_oracle(native, oracle, params):
    """Reads prepared on the GPU (translation, SEG, cutoffs) search exactly
    as the oracle's queries do."""
    db = W.make_database(1200, 75, median=250)
    reads = W.make_reads(db, 150, 76)
    codes, offs, lens, cut, trig = native.prepare_translated_queries(reads.dna, reads.offsets)
    q = W.translated_queries(codes, offs, lens, sources=reads.sources, cutoffs=(cut, trig))
    e = native.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        e.presearch(native.SCHEDULE_BATCHED)
        got = e.results()
        res, cnt, _ = oracle.presearch(params, db, q)
        assert cnt["gapped_extensions"] > 0
        for i in range(q.number):
            assert np.array_equal(got[i], res[i]), i
    finally:
        e.close()


@pytest.mark.parametrize("filter_", [True, False])
def test_engine_prepares_protein_queries_on_device(native, oracle, params, filter_):
    """gzb_engine_set_protein_queries (SEG, cutoffs and hash lists on the
    device, the prepared codes never read back) gives the cutoffs, lists and
    presearch results of prepare_protein_queries + set_queries, whose
    preparation the oracle pins; with the filter, short, low-complexity and
    lower-case proteins are mixed in."""
    rng = np.random.default_rng(91)
    db = W.make_database(1200, 93, median=250)
    seqs = W.query_sequences(W.make_queries(db, 150, 94, median=250))
    if filter_:
        seqs += [native.encode_protein_for_seg(_low_complexity_protein(rng, n))
                 for n in (0, 1, 5, 11, 12, 13, 50, 300, 900)]
    q = W.pack_queries(seqs, cutoffs=(np.zeros(len(seqs), np.int32),
                                      np.zeros(len(seqs), np.int32)))
    codes, cut, trig = native.prepare_protein_queries(q.codes, q.offsets, q.lengths,
                                                      filter=filter_)
    ref = W.Queries(codes=codes, offsets=q.offsets, lengths=q.lengths, cutoffs=cut,
                    triggers=trig)
    e = native.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(ref)
        lists_a = e.list_arrays()
        e.reset_results()
        e.presearch(native.SCHEDULE_BATCHED)
        res_a = e.results()
        cut_b, trig_b = e.set_protein_queries(q.codes, q.offsets, q.lengths, filter=filter_)
        assert np.array_equal(cut_b, cut) and np.array_equal(trig_b, trig)
        lists_b = e.list_arrays()
        for name in lists_a:
            assert np.array_equal(lists_a[name], lists_b[name]), name
        e.reset_results()
        e.presearch(native.SCHEDULE_BATCHED)
        res_b = e.results()
        assert sum(len(r) for r in res_a) > 0
        for i in range(q.number):
            assert np.array_equal(res_a[i], res_b[i]), i
        if filter_:
            exp, _, _ = oracle.presearch(params, db, ref)
            for i in range(q.number):
                assert np.array_equal(res_b[i], exp[i]), i
    finally:
        e.close()


@pytest.mark.parametrize("filter_", [True, False])
def test_engine_prepares_translated_queries_on_device(native, oracle, params, filter_):
    """gzb_engine_set_translated_queries (translation, SEG, cutoffs and hash
    lists on the device) gives the cutoffs, lists and presearch results of
    prepare_translated_queries + set_queries, on reads with N, lower case,
    short reads and tandem repeats mixed into reads of the database."""
    rng = np.random.default_rng(95)
    db = W.make_database(1200, 97, median=250)
    reads = W.make_reads(db, 120, 98)
    extra, extra_dna, extra_off = _reads(rng, 40)
    dna = np.concatenate([reads.dna, extra_dna]).astype(np.uint8)
    offsets = np.concatenate([reads.offsets, reads.offsets[-1] + extra_off[1:]]).astype(np.uint64)
    codes, offs, lens, cut, trig = native.prepare_translated_queries(dna, offsets,
                                                                     filter=filter_)
    ref = W.translated_queries(codes, offs, lens, cutoffs=(cut, trig))
    e = native.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(ref)
        lists_a = e.list_arrays()
        e.reset_results()
        e.presearch(native.SCHEDULE_BATCHED)
        res_a = e.results()
        cut_b, trig_b = e.set_translated_queries(dna, offsets, filter=filter_)
        assert np.array_equal(cut_b, cut) and np.array_equal(trig_b, trig)
        lists_b = e.list_arrays()
        for name in lists_a:
            assert np.array_equal(lists_a[name], lists_b[name]), name
        e.reset_results()
        e.presearch(native.SCHEDULE_BATCHED)
        res_b = e.results()
        assert sum(len(r) for r in res_a) > 0
        for i in range(ref.number):
            assert np.array_equal(res_a[i], res_b[i]), i
    finally:
        e.close()
