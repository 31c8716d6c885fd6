"""The `aln` tabular lines (AlignerCommon::WriteOutput,
src/aligner_common.h:344-394) written on the host from alignment records,
without a device: field by field against values computed from the
reference's own hit statistics and read coordinates (its compiled units),
for protein and translated queries."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W


def _records(rng, db, n):
    from gzb import native as N
    r = np.zeros(n, N.ALIGNMENT_DTYPE)
    subj = rng.integers(0, db.number_sequences, n)
    first = db.offsets[subj].astype(np.int64)
    r["subject_id"] = subj
    r["score"] = rng.integers(20, 400, n)
    r["start_d"] = first + rng.integers(0, 30, n)
    r["end_d"] = r["start_d"] + rng.integers(5, 60, n)
    r["start_q"] = rng.integers(1, 40, n)
    r["end_q"] = r["start_q"] + rng.integers(5, 60, n)
    r["alignment_length"] = rng.integers(10, 80, n)
    r["mismatches"] = rng.integers(0, 10, n)
    r["gap_openings"] = rng.integers(0, 3, n)
    r["gap_extensions"] = r["gap_openings"] + rng.integers(0, 3, n)
    return r


@pytest.mark.parametrize("translated", [False, True])
def test_hit_table_lines(reference, translated):
    from gzb import native as N
    params = P.make_params()
    rng = np.random.default_rng(91 + translated)
    db = W.make_database(50, 93, median=120)
    db_len = int(db.length - db.number_sequences - 1)
    n_queries = 6
    results = [_records(rng, db, int(rng.integers(0, 6))) for _ in range(n_queries)]
    dna = rng.integers(150, 400, n_queries) if translated else None
    real = dna // 3 if translated else rng.integers(50, 500, n_queries)
    qn = [f"q{i}" for i in range(n_queries)]
    sn = [f"s{j}" for j in range(db.number_sequences)]
    lines = N.hit_table(results, qn, sn, db.offsets, db_len, db.number_sequences, real,
                        dna_lengths=dna)
    assert len(lines) == sum(len(r) for r in results) > 0
    it = iter(lines)
    for qi, rows in enumerate(results):
        for r in rows:
            f = next(it).split("\t")
            assert f[0] == qn[qi] and f[1] == sn[int(r["subject_id"])]
            diff = np.float32(r["mismatches"] + r["gap_openings"] + r["gap_extensions"])
            ident = (1.0 - float(diff / np.float32(r["alignment_length"]))) * 100
            assert f[2] == "%g" % ident
            assert [int(x) for x in f[3:6]] == [int(r["alignment_length"]), int(r["mismatches"]),
                                                int(r["gap_openings"])]
            sq, eq = int(r["start_q"]), int(r["end_q"])
            if translated:
                sq = reference.translated_real(params, b"A" * int(dna[qi]), sq)[0]
                eq = reference.translated_real(params, b"A" * int(dna[qi]), eq)[1]
            assert [int(f[6]), int(f[7])] == [sq, eq]
            first = int(db.offsets[int(r["subject_id"])]) - 1
            assert [int(f[8]), int(f[9])] == [int(r["start_d"]) - first, int(r["end_d"]) - first]
            _, ev, bs = reference.hit_statistics(params, int(real[qi]), db_len,
                                                 db.number_sequences, int(r["score"]))
            assert abs(float(f[10]) - ev) <= 1e-9 * ev or f[10] == "%g" % ev
            assert f[10] == "%g" % ev and f[11] == "%g" % bs
