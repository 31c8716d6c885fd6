"""Pins the C restatement (oracle/gz_oracle.c) to the reference: the
reference's own units compiled from its sources (oracle/_ref) on random
inputs, and the known answers of the reference's unit tests."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

DNA_DELIM = 5  # "ACGT" + unknown N -> max code 4, delimiter 5


def dna(s):
    return np.array([DNA_DELIM] + ["ACGT".index(c) for c in s] + [DNA_DELIM], np.uint8)


def dna_params():
    """match 2 / mismatch -1 over 4 letters (test/gapped_extender_test.cpp:24-46)."""
    m = np.full((4, 4), -1, np.int32)
    np.fill_diagonal(m, 2)
    p = P.make_params(matrix=m, gap_open=0, gap_extension=1)
    p["delimiter"] = DNA_DELIM
    return p


# --- known answers of the reference unit tests ------------------------------
def test_gapped_known_answer_cpu(oracle):
    # test/gapped_extender_test.cpp:49-56: AGTCAC vs AGCAG, forward from the
    # first residue, open 0 / extend 1, no X-drop -> 7 at (4, 3)
    p = dna_params()
    s0, s1 = dna("AGTCAC"), dna("AGCAG")
    score, q, d, _ = oracle.gapped_one_side(p, s0, 1, s1, 1, False, 2**31 - 1)
    assert (score, q, d) == (7, 4, 3)


def test_gapped_known_answers_gpu_suite(oracle):
    # test/gapped_extender_gpu_test.cu:40-253 (absolute positions returned)
    p = dna_params()
    s0, s1 = dna("AGCAC"), dna("AGCAG")
    score, q, d, _ = oracle.gapped_one_side(p, s0, 1, s1, 1, False, 0)
    assert (score, 1 + q, 1 + d) == (8, 4, 4)
    s0, s1 = dna("AGTCAC"), dna("AGCAG")
    score, q, d, _ = oracle.gapped_one_side(p, s0, 1, s1, 1, False, 2**31 - 1)
    assert (score, 1 + q, 1 + d) == (7, 5, 4)
    score, q, d, _ = oracle.gapped_one_side(p, s0, len(s0) - 3, s1, len(s1) - 3, True,
                                            2**31 - 1)
    assert (score, len(s0) - 3 + q, len(s1) - 3 + d) == (7, 1, 1)


def test_ungapped_known_answers(oracle):
    # test/ungapped_extender_test.cpp:18-114
    p = dna_params()
    s0, s1 = dna("AAAAAAC"), dna("AACAAAG")
    fwd = oracle.ungapped_one_side(p, s0, 1, s1, 1, False, 2**31 - 1)
    rev = oracle.ungapped_one_side(p, s0, len(s0) - 3, s1, len(s1) - 3, True, 2**31 - 1)
    assert fwd == 9 and rev == fwd
    assert oracle.ungapped_one_side(p, s0, 1, s1, 1, False, 1) == 4


def test_distance_known_answers(oracle, params):
    # test/distance_calculator_test.cpp:56-117 (L = 4, centres 2/6/10)
    p = params.copy()
    p["subsequence_length"] = 4
    a = P.encode("IMEHQSIMEHQS")
    b = P.encode("LMEHQALMEHQA")
    assert [oracle.distance(p, a, c, b, c) for c in (2, 6, 10)] == [0, 1, 1]
    p["subsequence_length"] = 6
    assert oracle.distance(p, P.encode("GMEHQS"), 3, P.encode("GMEHQS"), 3) == 0
    assert oracle.distance(p, P.encode("IMEHQS"), 3, P.encode("LMEHQA"), 3) == 1


def test_chain_filter_known_answers(oracle):
    # test/chain_filter_test.cpp:11-121
    p = dna_params()
    q = dna("AAAAAAC")
    assert len(oracle.chain_filter(p, q, len(q), 1, dna("AAACAAG"), [1, 3], [1, 3])[0]) == 1
    assert len(oracle.chain_filter(p, q, len(q), 1, dna("AACAAAG"), [1, 2], [1, 2])[0]) == 1
    assert len(oracle.chain_filter(p, q, len(q), 1, dna("AACAAAG"), [1, 4], [1, 4])[0]) == 2


def test_hash_known_answer(oracle, params):
    # test/reduced_alphabet_variable_hash_function_test.cpp:104-127 idea:
    # the hash of a k-mer is its reduced codes (+1) packed 4 bits each until
    # the code-score sum reaches the threshold (6..8 codes).
    rmap, _ = P.reduced_code_map()
    seq = np.concatenate([P.encode("GMEHQSWWCC"), [P.DELIMITER]]).astype(np.uint8)
    r, h, ln = oracle.hash(params, seq)
    exp_h, score, k = 0, 0, 0
    while k < 8 and not (k >= 6 and score >= 39):
        c = int(rmap[seq[k]])
        exp_h = (exp_h << 4) + c + 1
        score += int(params["code_scores"][c])
        k += 1
    assert (r, h, ln) == (0, exp_h, k)


# --- random differential against the reference's own units ------------------
def _seq_with_noise(rng, n):
    s = W.random_residues(rng, n)
    noise = rng.random(n)
    s[noise < 0.02] = 24  # X
    s[(noise >= 0.02) & (noise < 0.03)] = 20  # B
    s[(noise >= 0.03) & (noise < 0.05)] = P.DELIMITER
    return s


def test_hash_matches_reference(oracle, reference, params):
    rng = np.random.default_rng(7)
    seq = np.concatenate([[25], _seq_with_noise(rng, 20000), [25] * 16]).astype(np.uint8)
    r, h, ln = reference.hash_many(params, seq)
    for i in range(0, len(r), 7):
        rr, hh, ll = oracle.hash(params, seq, i)
        assert rr == r[i]
        if rr == 0:
            assert (hh, ll) == (h[i], ln[i])


def test_distance_matches_reference(oracle, reference, params):
    rng = np.random.default_rng(8)
    a = W.random_residues(rng, 5000)
    b = a.copy()
    mut = rng.random(len(b)) < 0.2
    b[mut] = W.random_residues(rng, int(mut.sum()))
    c0 = rng.integers(5, 4990, 2000).astype(np.uint32)
    c1 = np.clip(c0.astype(np.int64) + rng.integers(-3, 4, 2000), 5, 4990).astype(np.uint32)
    ref = reference.distances(params, a, b, c0, c1)
    mine = [oracle.distance(params, a, int(x), b, int(y)) for x, y in zip(c0, c1)]
    assert np.array_equal(ref, np.array(mine, np.int8))


def _pair(rng, n, ident):
    a = W.random_residues(rng, n)
    b = W.mutate(rng, a, ident)
    return (np.concatenate([[25], a, [25]]).astype(np.uint8),
            np.concatenate([[25], b, [25]]).astype(np.uint8))


def test_ungapped_matches_reference(oracle, reference, params):
    rng = np.random.default_rng(9)
    for t in range(400):
        a, b = _pair(rng, int(rng.integers(5, 300)), rng.uniform(0.2, 1.0))
        pa = int(rng.integers(1, len(a) - 1))
        pb = int(rng.integers(1, len(b) - 1))
        cutoff = int(rng.integers(1, 40))
        for rev in (False, True):
            assert oracle.ungapped_one_side(params, a, pa, b, pb, rev, cutoff) == \
                reference.ungapped_one_side(params, a, pa, b, pb, rev, cutoff)


@pytest.mark.parametrize("seed", [10, 11, 12])
def test_gapped_matches_reference(oracle, reference, params, seed):
    rng = np.random.default_rng(seed)
    for t in range(150):
        a, b = _pair(rng, int(rng.integers(5, 600)), rng.uniform(0.25, 1.0))
        pa = int(rng.integers(1, len(a) - 1))
        pb = int(np.clip(pa + rng.integers(-5, 6), 1, len(b) - 2))
        cutoff = int(rng.choice([0, 5, 15, 26, 40, 2**31 - 1]))
        for rev in (False, True):
            len0 = pa if rev else len(a) - pa
            r = reference.gapped_one_side(params, a, pa, len0, b, pb, rev, cutoff)
            m = oracle.gapped_one_side(params, a, pa, b, pb, rev, cutoff)[:3]
            assert m == r, (t, rev, cutoff)


def test_chain_filter_matches_reference(oracle, reference, params):
    rng = np.random.default_rng(13)
    for t in range(100):
        a, b = _pair(rng, int(rng.integers(30, 400)), rng.uniform(0.4, 1.0))
        n = int(rng.integers(1, 60))
        diag = int(rng.integers(-5, 6))
        hq = rng.integers(1, len(a) - 1, n)
        hd = np.clip(hq + diag + rng.integers(-1, 2, n) * rng.integers(0, 2, n), 1, len(b) - 2)
        # unique (q, d) pairs, as seeds are
        pairs = sorted(set(zip(hq.tolist(), hd.tolist())))
        hq = [x for x, _ in pairs]
        hd = [y for _, y in pairs]
        cutoff = int(rng.integers(1, 30))
        rq, rd = reference.chain_filter(params, a, len(a), cutoff, b, hq, hd)
        mq, md = oracle.chain_filter(params, a, len(a), cutoff, b, hq, hd)
        assert sorted(zip(rq.tolist(), rd.tolist())) == sorted(zip(mq.tolist(), md.tolist()))
        assert list(md) == sorted(md)


def test_db_index_matches_reference(oracle, reference, params):
    db = W.make_database(300, 21, median=120)
    mine = oracle.db_index(params, db.codes)
    h = reference.db_index(params, db.codes)
    try:
        # every hash of the database is either in the residual index, the
        # representative index, or absent from both, exactly as in the reference
        keys = set(mine["nc_keys"].tolist()) | set(mine["rep_keys"].tolist())
        for k in range(len(mine["nc_keys"])):
            key = int(mine["nc_keys"][k])
            v = mine["nc_values"][mine["nc_offsets"][k]:mine["nc_offsets"][k + 1]]
            assert np.array_equal(reference.lookup(h, 0, key), v)
        ref_cluster_members = {}
        for k in range(len(mine["rep_keys"])):
            key = int(mine["rep_keys"][k])
            lo, hi = mine["rep_offsets"][k], mine["rep_offsets"][k + 1]
            r = reference.lookup(h, 1, key).reshape(-1, 2)
            assert np.array_equal(r[:, 1], mine["rep_positions"][lo:hi])
            for (rcid, _), cid in zip(r, mine["rep_cluster_ids"][lo:hi]):
                mm = mine["member_positions"][mine["member_offsets"][cid]:mine["member_offsets"][cid + 1]]
                assert np.array_equal(reference.members(h, int(rcid)), mm)
        r_, hh, _ = reference.hash_many(params, np.concatenate([db.codes, [25] * 16]).astype(np.uint8))
        for key in set(hh[r_ == 0].tolist()) - keys:
            assert len(reference.lookup(h, 0, key)) == 0
            assert len(reference.lookup(h, 1, key)) == 0
        assert len(mine["rep_keys"]) > 0 and len(mine["member_positions"]) > 0
    finally:
        reference.free_index(h)


def test_cutoffs_match_reference(reference, params):
    rng = np.random.default_rng(14)
    for _ in range(100):
        s = W.random_residues(rng, int(rng.integers(20, 1000)))
        lam, k, _ = reference.ungapped_karlin(params, np.concatenate([[25], s, [25]]))
        ml, mk, _ = P.ungapped_karlin_for_query(s)
        assert (np.float32(ml), np.float32(mk)) == (np.float32(lam), np.float32(k))
        assert reference.cutoffs(lam, k) == (P.normalized_cutoff_to_nominal(7.0, ml),
                                             P.normalized_to_nominal(22.0, ml, mk))


# --- traceback (build results) ------------------------------------------------
def test_edit_path_known_answer(oracle):
    # test/gapped_extender_test.cpp:49-94: AGTCAC vs AGCAG, forward, open 0 /
    # extend 1, no X-drop -> 7 at (4, 3) with path S S G1 S S
    p = dna_params()
    s0, s1 = dna("AGTCAC"), dna("AGCAG")
    score, q, d, ops = oracle.gapped_one_side_edits(p, s0, 1, s1, 1, False, 2**31 - 1)
    assert (score, q, d) == (7, 4, 3)
    assert list(ops[:5]) == [1, 1, 2, 1, 1]


@pytest.mark.parametrize("seed", [20, 21])
def test_edit_path_matches_reference(oracle, reference, params, seed):
    rng = np.random.default_rng(seed)
    for t in range(120):
        a, b = _pair(rng, int(rng.integers(5, 500)), rng.uniform(0.25, 1.0))
        pa = int(rng.integers(1, len(a) - 1))
        pb = int(np.clip(pa + rng.integers(-5, 6), 1, len(b) - 2))
        cutoff = int(rng.choice([0, 5, 15, 26, 40, 2**31 - 1]))
        for rev in (False, True):
            len0 = pa if rev else len(a) - pa
            r = reference.gapped_one_side_edits(params, a, pa, len0, b, pb, rev, cutoff)
            m = oracle.gapped_one_side_edits(params, a, pa, b, pb, rev, cutoff)
            assert m[:3] == r[:3], (t, rev, cutoff)
            assert np.array_equal(m[3], r[3]), (t, rev, cutoff)
            # same score and end point as the score-only extension
            assert m[:3] == oracle.gapped_one_side(params, a, pa, b, pb, rev, cutoff)[:3]


def test_alignment_statistics_by_hand(oracle):
    # forward path S S G1 S S after a reverse side that stops at once: the
    # alignment AG-CA against AGTCA (query AGTCAC, hit at its first residue)
    p = dna_params()
    p["gapped_cutoff"] = 2**31 - 1
    q, d = dna("AGTCAC"), dna("AGCAG")
    a = oracle.build_alignment(p, q, 1, d, 1)
    assert (a["score"], a["start_q"], a["start_d"], a["end_q"], a["end_d"]) == (7, 1, 1, 5, 4)
    assert (a["alignment_length"], a["mismatches"], a["gap_openings"],
            a["gap_extensions"]) == (5, 0, 1, 0)


# --- six-frame translation (query preparation) -------------------------------
def _frames(codes, length):
    """Split a translated query into its six frames (codes between the
    frame delimiters)."""
    slot = length // 3 + 1
    out = []
    for f in range(6):
        s = codes[1 + f * slot: 1 + (f + 1) * slot]
        out.append("".join(P.LETTERS[c] for c in s if c != P.DELIMITER))
    return out


def test_translation_known_answers(oracle):
    # test/translator_test.cpp:22-43
    read = b"GCCCGCCACCT"
    q = oracle.translate_query(read, P.DELIMITER)
    assert len(q) == 7 + 6 * 3
    assert _frames(q, len(read)) == ["ARH", "PAT", "PPP", "RWR", "GGG", "VAG"]
    read = b"GCCCGCCACC"
    q = oracle.translate_query(read, P.DELIMITER)
    assert _frames(q, len(read)) == ["ARH", "PAT", "PP", "GGG", "VAG", "WR"]
    # a frame short of length/3 codons carries an extra delimiter
    assert list(q[1 + 2 * 4 + 2:1 + 3 * 4]) == [P.DELIMITER, P.DELIMITER]


def test_translation_frame_layout(oracle):
    # test/translated_dna_query_test.cpp:29-31, :67-90: a 75-base read has
    # 26-code frame slots, so position 27 opens frame 1 and 79 opens frame 3
    read = b"AGCGAGAGCGAGTGGTGGGCAAAAAAACCTATACTGCAAAATTTTATGAAAGGTGCTTATTGTCCTCTGAATGAT"
    q = oracle.translate_query(read, P.DELIMITER)
    assert len(q) == 7 + 6 * 25
    assert all(q[1 + 26 * f - 1] == P.DELIMITER for f in range(7))
    assert q[27] != P.DELIMITER and q[79] != P.DELIMITER


def test_translation_reverse_frames_are_complement_strand(oracle):
    # test/test_dna.fa: test7 is the reverse complementary strand of test6
    # (also test/dna_sequence_test.cpp:19-23)
    t6 = b"GCTGCTGCTGCTGCTGCTGCTGCTGCTGCTGCTGCTGCTGCTGCTATGAAAGGTGCTTATTGTCCTCTGAATGAT"
    t7 = b"ATCATTCAGAGGACAATAAGCACCTTTCATAGCAGCAGCAGCAGCAGCAGCAGCAGCAGCAGCAGCAGCAGCAGC"
    f6 = _frames(oracle.translate_query(t6, P.DELIMITER), len(t6))
    f7 = _frames(oracle.translate_query(t7, P.DELIMITER), len(t7))
    assert f6[3:] == f7[:3] and f6[:3] == f7[3:]


def test_translation_short_reads(oracle):
    for read in (b"", b"A", b"AC"):
        assert list(oracle.translate_query(read, P.DELIMITER)) == [P.DELIMITER] * 2


def _random_read(rng, n):
    # mostly ACGT with some N, lowercase and other IUPAC letters
    letters = np.frombuffer(b"ACGTACGTACGTACGTacgtNNRYKM", np.uint8)
    return bytes(letters[rng.integers(0, len(letters), n)])


@pytest.mark.parametrize("seed", [30, 31])
def test_translation_matches_reference(oracle, reference, params, seed):
    rng = np.random.default_rng(seed)
    for t in range(300):
        n = int(rng.choice([3, 4, 5, 6, 7, 8, 150, int(rng.integers(3, 2000))]))
        read = _random_read(rng, n)
        r = reference.translate_query(params, read)
        m = oracle.translate_query(read, params["delimiter"])
        assert np.array_equal(m, r), (t, n)


def test_translated_query_cutoffs_match_reference(oracle, reference, params):
    # TranslatedDnaQuery::SetStaticalParameters (src/translated_dna_query.cpp:76-85)
    # takes the composition of the whole translated query: delimiters, stop
    # codons and unknown codons included
    db = W.make_database(50, 33)
    reads = W.make_reads(db, 60, 34)
    for r in range(reads.number):
        q = oracle.translate_query(reads.read(r), params["delimiter"])
        lam, k, _ = reference.ungapped_karlin(params, q)
        ml, mk, _ = P.ungapped_karlin_for_query(q[1:-1])
        assert (np.float32(ml), np.float32(mk)) == (np.float32(lam), np.float32(k))
        cut, trig = P.query_cutoffs([q[1:-1]])
        assert reference.cutoffs(lam, k) == (int(cut[0]), int(trig[0]))


# --- per-query Karlin statistics (query preparation) ---------------------------
def test_query_karlin_matches_reference(oracle, reference, params):
    # Statistics::CalculateUngappedKarlinParameters (src/statistics.cpp:205-229)
    # and the cutoffs of src/aligner_gpu.cpp:228-238, on protein queries,
    # translated queries and skewed short compositions
    rng = np.random.default_rng(35)
    db = W.make_database(40, 36)
    reads = W.make_reads(db, 100, 37)
    cases = [np.concatenate([[25], W.random_residues(rng, int(rng.integers(5, 3000))), [25]])
             for _ in range(150)]
    cases += [oracle.translate_query(reads.read(r), 25) for r in range(reads.number)]
    for _ in range(150):
        letters = rng.choice(25, size=int(rng.integers(1, 6)), replace=False)
        body = rng.choice(letters, size=int(rng.integers(1, 400))).astype(np.uint8)
        cases.append(np.concatenate([[25], body, [25]]).astype(np.uint8))
    for n in (1000, 5000):  # poly-S: the K series needs 31-32 rounds
        cases.append(np.concatenate([[25], np.full(n, 15), [25]]).astype(np.uint8))
    for q in cases:
        lam, k, h = reference.ungapped_karlin(params, q)
        ol, ok, oh, cut, trig = oracle.query_karlin(params, q)
        assert (np.float32(ol), np.float32(ok), np.float32(oh)) == \
            (np.float32(lam), np.float32(k), np.float32(h)), q
        assert (cut, trig) == reference.cutoffs(lam, k)


# --- SEG low-complexity filter (query preparation) -----------------------------
def test_seg_ln_factorial_table_matches_reference(oracle):
    # ext/seg/src/ln_factrial_table.h: ln(n!) to 6 decimals, n = 0..10000,
    # read as text from the reference checkout the oracle's recipe uses
    import os
    import re
    import oracle as O
    if not O.REF_ROOT:
        pytest.skip("GZ_REFERENCE_ROOT (the reference checkout) not set")
    REF_LN_FACT = os.path.join(O.REF_ROOT, "ext", "seg", "src", "ln_factrial_table.h")
    if not os.path.exists(REF_LN_FACT):
        pytest.skip("reference checkout not present")
    text = open(REF_LN_FACT).read()
    body = text[text.index("{", text.index("kLnFactrialTable")) + 1:text.rindex("};")]
    vals = [float(v) for v in re.findall(r"[0-9]+\.[0-9]+", body)]
    assert len(vals) == 10001
    assert all(oracle.L.gzo_ln_factorial6(n) == v for n, v in enumerate(vals))


def _low_complexity_protein(rng, n):
    """Random protein letters with planted low-complexity stretches (repeats
    of 1-4 letters), stop and unknown letters, and some lower case."""
    letters = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", np.uint8)
    s = letters[rng.integers(0, 20, n)].copy()
    for _ in range(int(rng.integers(0, 4))):
        if n < 2:
            break
        a = int(rng.integers(0, n - 1))
        b = min(n, a + int(rng.integers(5, 60)))
        pool = letters[rng.choice(20, size=int(rng.integers(1, 5)), replace=False)]
        s[a:b] = pool[rng.integers(0, len(pool), b - a)]
    extra = rng.random(n)
    s[extra < 0.02] = ord("*")
    s[(extra >= 0.02) & (extra < 0.03)] = ord("X")
    low = (extra >= 0.03) & (extra < 0.035)
    s[low] = s[low] | 0x20
    s[s == ord("*") | 0x20] = ord("*")
    return bytes(s)


@pytest.mark.parametrize("seed", [60, 61])
def test_seg_mask_matches_reference(oracle, reference, seed):
    rng = np.random.default_rng(seed)
    masked_any = 0
    for t in range(400):
        n = int(rng.choice([0, 5, 11, 12, 13, 20, 50, int(rng.integers(12, 400)),
                            int(rng.integers(400, 2500))]))
        s = _low_complexity_protein(rng, n)
        r = reference.seg_mask(s)
        m = oracle.seg_mask(s)
        assert m == r, (t, n, s)
        masked_any += bool(m and b"x" in m)
    assert masked_any > 50


def test_seg_known_answer(oracle):
    # a poly-Q stretch (positions 21-46) inside a random protein: windows are
    # keyed by their first position, so the mask covers 21-44 and the last
    # two Q stay; everything else is kept (as the reference's seg does)
    s = b"MKTAYIAKQRQISFVKSHFSRQ" + b"Q" * 25 + b"LEERLGLIEVQAPILSRVGDGTQDNLSGAEKAVQVKVKALPDAQ"
    m = oracle.seg_mask(s)
    assert m == s[:21] + b"x" * 24 + s[45:]
    assert oracle.seg_mask(b"QQQQQQQQQQQ") is None  # shorter than the window


def test_translation_with_seg_matches_reference(oracle, reference, params):
    rng = np.random.default_rng(62)
    for t in range(300):
        n = int(rng.choice([3, 20, 35, 36, 37, 150, int(rng.integers(3, 1500))]))
        if rng.random() < 0.3:  # low-complexity DNA: short tandem repeats
            unit = bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(rng.integers(1, 7)))])
            read = (unit * (n // len(unit) + 1))[:n]
        else:
            read = _random_read(rng, n)
        r = reference.translate_query_seg(params, read)
        m = oracle.translate_query_seg(read, params["delimiter"])
        assert np.array_equal(m, r), (t, n, read)


def test_protein_query_with_seg_matches_reference(oracle, reference, params):
    # ProteinQuery with SEG (src/protein_query.cpp:39-58): masked codes and
    # the Karlin parameters of the whole held sequence, short proteins too
    rng = np.random.default_rng(63)
    for t in range(300):
        n = int(rng.choice([0, 1, 5, 11, 12, 13, int(rng.integers(12, 600))]))
        s = _low_complexity_protein(rng, n)
        r, rl, rk = reference.protein_query_seg(params, s)
        m = oracle.protein_query_seg(s, params["delimiter"])
        assert np.array_equal(m, r), (t, n, s)
        lam, k, _, _, _ = oracle.query_karlin(params, m)
        assert (np.float32(lam), np.float32(k)) == (np.float32(rl), np.float32(rk)), (t, n)


# --- the final hit table ----------------------------------------------------------
def test_hit_statistics_match_reference(oracle, reference, params):
    # Statistics::CalculateSearchSpace / Nominal2EValue / Nominal2Normalized
    # (src/statistics.cpp:23-122) as AlignerCommon::WriteOutput uses them
    rng = np.random.default_rng(80)
    cases = [(300, 719856279, 2000000), (50, 5762314777, 16000000), (1, 1000, 10),
             (8000, 71906369, 200000), (12, 36, 3), (150, 1000000, 1)]
    cases += [(int(rng.integers(1, 10000)), int(rng.integers(1, 10**10)),
               int(rng.integers(1, 10**7))) for _ in range(200)]
    for ql, dl, ns in cases:
        if ns > dl:
            ns = dl
        for score in (0, 1, 38, 57, int(rng.integers(20, 3000))):
            exp = reference.hit_statistics(params, ql, dl, ns, score)
            got = oracle.hit_statistics(ql, dl, ns, score)
            assert got[0] == exp[0] and got[1] == exp[1], (ql, dl, ns, score, got, exp)
            assert np.float32(got[2]) == np.float32(exp[2])


def test_translated_coordinates_match_reference(oracle, reference, params):
    # TranslatedDnaQuery::GetRealStart / GetRealEnd (src/translated_dna_query.h:43-61)
    rng = np.random.default_rng(81)
    for n in (3, 4, 5, 75, 150, 151, 152, 1000):
        read = bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, n)])
        slot = n // 3 + 1
        for f in range(6):
            for j in range(0, slot - 1):
                pos = 1 + f * slot + j
                assert oracle.translated_real(pos, n) == reference.translated_real(params, read, pos)
