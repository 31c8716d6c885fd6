"""The final hit table (the `aln` tabular output of
AlignerCommon::WriteOutput, src/aligner_common.h:344-394) built from the
GPU's presearch and build results step, against one built from the
oracle's presearch, alignments and hit statistics, for protein and for
translated queries (read coordinates).  E-values must match to 1e-9
relative (they match exactly)."""
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


def _expected(oracle, params, db, q, real_lengths, dna_lengths, q_names, s_names,
              db_length, db_sequences):
    res = oracle.presearch(params, db, q)[0]
    rows = []
    for qi in range(q.number):
        off = int(q.offsets[qi])
        for r in res[qi]:
            a = oracle.build_alignment(params, q.codes, off + int(r["hit_q"]), db.codes,
                                       int(r["hit_d"]))
            _, ev, bs = oracle.hit_statistics(int(real_lengths[qi]), db_length, db_sequences,
                                              a["score"])
            diff = np.float32(a["mismatches"] + a["gap_openings"] + a["gap_extensions"])
            ident = (1.0 - float(diff / np.float32(a["alignment_length"]))) * 100
            sq, eq = a["start_q"] - off, a["end_q"] - off
            if dna_lengths is not None:
                sq = oracle.translated_real(sq, int(dna_lengths[qi]))[0]
                eq = oracle.translated_real(eq, int(dna_lengths[qi]))[1]
            first = int(db.offsets[int(r["subject_id"])]) - 1
            rows.append((q_names[qi], s_names[int(r["subject_id"])], ident,
                         a["alignment_length"], a["mismatches"], a["gap_openings"], sq, eq,
                         a["start_d"] - first, a["end_d"] - first, ev, bs))
    return rows


def _compare(lines, rows):
    assert len(lines) == len(rows) and len(rows) > 0
    for line, row in zip(lines, rows):
        f = line.split("\t")
        assert f[0] == row[0] and f[1] == row[1]
        assert f[2] == "%g" % row[2]
        assert [int(x) for x in f[3:10]] == [int(x) for x in row[3:10]]
        ev = float(f[10])
        assert abs(ev - row[10]) <= 1e-9 * abs(row[10]) + 1e-300 or f[10] == "%g" % row[10]
        assert f[10] == "%g" % row[10] and f[11] == "%g" % row[11]


def test_protein_hit_table(native, oracle, params):
    N = native
    db = W.make_database(1500, 3101, median=250)
    q = W.make_queries(db, 120, 3102, median=250)
    q_names = [f"query{i}" for i in range(q.number)]
    s_names = [f"subject{j}" for j in range(db.number_sequences)]
    real = q.lengths.astype(np.int64) - 2
    db_len = int(db.length - db.number_sequences - 1)  # residues, no delimiters
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        e.set_graph(True)
        e.presearch(N.SCHEDULE_BATCHED)
        lines = N.hit_table(e.build_alignments(), q_names, s_names, db.offsets, db_len,
                            db.number_sequences, real)
    finally:
        e.close()
    _compare(lines, _expected(oracle, params, db, q, real, None, q_names, s_names, db_len,
                              db.number_sequences))


def test_translated_hit_table(native, oracle, params):
    N = native
    db = W.make_database(1200, 3103, median=250)
    reads = W.make_reads(db, 150, 3104)
    codes, offs, lens, cut, trig = N.prepare_translated_queries(reads.dna, reads.offsets)
    q = W.translated_queries(codes, offs, lens, cutoffs=(cut, trig))
    dna_lengths = np.diff(reads.offsets).astype(np.int64)
    real = dna_lengths // 3
    q_names = [f"read{i}" for i in range(q.number)]
    s_names = [f"protein{j}" for j in range(db.number_sequences)]
    db_len = int(db.length - db.number_sequences - 1)
    e = N.PresearchEngine(0)
    try:
        e.set_params(params)
        e.set_database(db)
        e.set_queries(q)
        e.presearch(N.SCHEDULE_BATCHED)
        lines = N.hit_table(e.build_alignments(), q_names, s_names, db.offsets, db_len,
                            db.number_sequences, real, dna_lengths=dna_lengths)
    finally:
        e.close()
    _compare(lines, _expected(oracle, params, db, q, real, dna_lengths, q_names, s_names,
                              db_len, db.number_sequences))
