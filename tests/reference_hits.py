"""Golden hit tables of the reference's own search, and the inputs they were
made from (test infrastructure).

Each case under tests/golden/reference_hits/ holds the tabular output of
the reference's GPU aligner (`ghostz-gpu aln -g 1`, its host code compiled
unchanged with CPU stand-ins for its device operators: oracle/ref_aln.py)
for a seeded synthetic workload, or for the reference's own example files
(data/db.fasta, data/queries.fasta, stored in the case).  The generating
script is tests/golden/make_reference_hit_tables.py.

This module rebuilds a case's inputs in the engine's layout (the database
split into the chunks the reference's `db` command made) and writes the
hit table two ways: through the CPU oracle's restatement of the path
(`oracle_hit_table`), and through the library's GPU search
(`engine_hit_table`, gzb/search.py).
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from gzb import params as P
from gzb import workload as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_hits")

# Every case: how its inputs are made.  "protein" / "reads" workloads come
# from the seeded generators (gzb/workload.py) with config-1 shapes; "fasta"
# cases carry their files.
CASES = {
    "readme": dict(kind="fasta", query_type="d"),
    "protein-1k-x-20k": dict(kind="protein", db=(20000, 101), queries=(1000, 102)),
    "protein-300-x-20k-4chunks": dict(kind="protein", db=(20000, 101), queries=(300, 103),
                                      chunk_bytes=2_000_000),
    "translated-2k-reads-x-20k": dict(kind="reads", db=(20000, 101), reads=(2000, 302)),
    "protein-200-x-5k-no-clustering": dict(kind="protein", db=(5000, 111), queries=(200, 112),
                                           clustering=False),
}


def read_fasta(text: str):
    """FastaSequenceReader::Read (src/fasta_sequence_reader.cpp:26-74): the
    name is the header after its leading '>' and spaces (a trailing '\\r'
    dropped, trailing spaces kept); sequence lines are trimmed, joined and
    upper-cased."""
    names, seqs = [], []
    for line in text.split("\n"):
        if line.startswith(">"):
            if line.endswith("\r"):
                line = line[:-1]
            names.append(line.lstrip("> "))
            seqs.append([])
        elif line.strip() and names:
            seqs[-1].append(line.strip())
    return names, ["".join(s).upper().encode() for s in seqs]


def fasta_text(names, seqs, width=60) -> bytes:
    out = []
    for name, seq in zip(names, seqs):
        out.append(b">" + name.encode() + b"\n")
        for i in range(0, max(len(seq), 1), width):
            out.append(bytes(seq[i:i + width]) + b"\n")
    return b"".join(out)


@dataclass
class CaseInputs:
    query_type: str                   # "p" protein or "d" DNA reads
    query_names: List[str]
    query_sequences: List[bytes]      # letters, or bases of reads
    subject_names: List[str]
    subject_sequences: List[bytes]    # letters
    clustering: bool = True
    chunk_bytes: Optional[int] = None

    def fasta(self):
        return (fasta_text(self.subject_names, self.subject_sequences),
                fasta_text(self.query_names, self.query_sequences))

    def sha256(self) -> str:
        db, q = self.fasta()
        return hashlib.sha256(db + b"\0" + q).hexdigest()


def case_inputs(name: str, stored: Optional[dict] = None) -> CaseInputs:
    spec = CASES[name]
    if spec["kind"] == "fasta":
        meta = stored if stored is not None else load_meta(name)
        qn, qs = read_fasta(meta["queries_fasta"])
        sn, ss = read_fasta(meta["db_fasta"])
        return CaseInputs(spec["query_type"], qn, qs, sn, ss)
    db = W.make_database(*spec["db"])
    sn = [f"s{j}" for j in range(db.number_sequences)]
    ss = [_letters(db.codes[int(db.offsets[j]):int(db.offsets[j + 1]) - 1])
          for j in range(db.number_sequences)]
    if spec["kind"] == "protein":
        q = W.make_queries(db, *spec["queries"])
        qs = [_letters(s) for s in W.query_sequences(q)]
        qn = [f"q{i}" for i in range(q.number)]
        qt = "p"
    else:
        reads = W.make_reads(db, *spec["reads"])
        qs = [reads.read(i) for i in range(reads.number)]
        qn = [f"r{i}" for i in range(reads.number)]
        qt = "d"
    return CaseInputs(qt, qn, qs, sn, ss, clustering=spec.get("clustering", True),
                      chunk_bytes=spec.get("chunk_bytes"))


def _letters(codes) -> bytes:
    return np.frombuffer(P.LETTERS.encode(), np.uint8)[np.asarray(codes, np.int64)].tobytes()


def load_meta(name: str) -> dict:
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)


def load_table(name: str) -> List[str]:
    with gzip.open(os.path.join(GOLDEN, name + ".tsv.gz"), "rt", encoding="latin-1") as f:
        return f.read().splitlines()


def database_chunks(inputs: CaseInputs, chunk_counts: List[int]) -> List[W.Database]:
    """The subjects split into chunks of the given sequence counts, each in
    the reference's chunk layout [delim s0 delim s1 ... delim]
    (src/database_chunk.h:282-300)."""
    chunks, at = [], 0
    for n in chunk_counts:
        seqs = [P.encode(s.decode("latin-1")) for s in inputs.subject_sequences[at:at + n]]
        lens = np.array([len(s) for s in seqs], np.int64)
        offsets = np.concatenate([[1], 1 + np.cumsum(lens + 1)]).astype(np.uint32)
        codes = np.full(int(offsets[-1]), P.DELIMITER, np.uint8)
        for s, o in zip(seqs, offsets[:-1]):
            codes[int(o):int(o) + len(s)] = s
        chunks.append(W.Database(codes=codes, offsets=offsets, number_sequences=n))
        at += n
    assert at == len(inputs.subject_sequences)
    return chunks


def case_params(inputs: CaseInputs):
    return P.make_params(clustering=inputs.clustering)


# -- the CPU oracle's composition ------------------------------------------------
def oracle_hit_table(oracle, inputs: CaseInputs, chunk_counts: List[int]) -> List[str]:
    """The hit table of the oracle's restatement: query preparation
    (gzo_protein_query_seg / gzo_translate_query_seg, gzo_query_karlin),
    each chunk's presearch merged in chunk order (gzo_add_results), the
    build results step (gzo_build_alignment), the reference's final order
    and line format."""
    p = case_params(inputs)
    delim = P.DELIMITER
    seqs, cut, trig, dna_len = [], [], [], []
    for s in inputs.query_sequences:
        c = (oracle.translate_query_seg(s, delim) if inputs.query_type == "d"
             else oracle.protein_query_seg(s, delim))
        k = oracle.query_karlin(p, c)
        seqs.append(c)
        cut.append(k[3])
        trig.append(k[4])
        dna_len.append(len(s))
    if inputs.query_type == "d":
        # translated queries hold their own delimiters between frames
        lens = np.array([len(c) for c in seqs], np.uint32)
        offs = np.concatenate([[0], np.cumsum(lens - 1)[:-1]]).astype(np.uint32)
        codes = np.zeros(int((lens - 1).sum()) + 1, np.uint8)
        for c, o in zip(seqs, offs):
            codes[int(o):int(o) + len(c)] = c
        q = W.Queries(codes=codes, offsets=offs, lengths=lens,
                      cutoffs=np.array(cut, np.int32), triggers=np.array(trig, np.int32))
        real = [n // 3 for n in dna_len]
    else:
        q = W.pack_queries([c[1:-1] for c in seqs],
                           cutoffs=(np.array(cut, np.int32), np.array(trig, np.int32)))
        real = [len(c) - 2 for c in seqs]
    chunks = database_chunks(inputs, chunk_counts)
    merged = [np.zeros(0, dtype=None) for _ in range(q.number)]
    for k, db in enumerate(chunks):
        res = oracle.presearch(p, db, q)[0]
        for qi in range(q.number):
            r = res[qi].copy()
            r["chunk_id"] = k
            merged[qi] = r if k == 0 else oracle.add_results(p, db, r, merged[qi])
    base = np.concatenate([[0], np.cumsum([db.number_sequences for db in chunks])])
    db_length = sum(int(db.length) - db.number_sequences - 1 for db in chunks)
    db_sequences = int(base[-1])
    lines = []
    for qi in range(q.number):
        off = int(q.offsets[qi])
        rows = []
        for r in merged[qi]:
            k = int(r["chunk_id"])
            db = chunks[k]
            a = oracle.build_alignment(p, q.codes, off + int(r["hit_q"]), db.codes,
                                       int(r["hit_d"]))
            _, ev, bs = oracle.hit_statistics(real[qi], db_length, db_sequences, a["score"])
            sq, eq = a["start_q"] - off, a["end_q"] - off
            if inputs.query_type == "d":
                sq = oracle.translated_real(sq, dna_len[qi])[0]
                eq = oracle.translated_real(eq, dna_len[qi])[1]
            first = int(db.offsets[int(r["subject_id"])]) - 1
            sd, ed = a["start_d"] - first, a["end_d"] - first
            diff = np.float32(a["mismatches"] + a["gap_openings"] + a["gap_extensions"])
            ident = (1.0 - float(diff / np.float32(a["alignment_length"]))) * 100
            name = inputs.subject_names[int(base[k]) + int(r["subject_id"])]
            rows.append((a["score"], (eq - sq) & 0xFFFFFFFF, (ed - sd) & 0xFFFFFFFF, sd,
                         "%s\t%s\t%g\t%d\t%d\t%d\t%d\t%d\t%d\t%d\t%g\t%g" % (
                             inputs.query_names[qi], name, ident, a["alignment_length"],
                             a["mismatches"], a["gap_openings"], sq, eq, sd, ed, ev, bs)))
        # AlignerBuildResultsThread::Run's final sort with ResultGreaterScore
        # (at most b rows: the insertion sort std::sort uses, which keeps ties)
        rows.sort(key=lambda x: (-x[0], -x[1], -x[2], x[3]))
        lines += [x[4] for x in rows]
    return lines


# -- the library's GPU search ------------------------------------------------------
def engine_hit_table(inputs: CaseInputs, chunk_counts: List[int], schedule=None,
                     graph=False) -> List[str]:
    from gzb import native as N
    from gzb import search as S
    p = case_params(inputs)
    if inputs.query_type == "d":
        dna = np.frombuffer(b"".join(inputs.query_sequences), np.uint8)
        offsets = np.concatenate([[0], np.cumsum([len(s) for s in inputs.query_sequences])])
        prepared = S.translated_queries(dna, offsets.astype(np.uint64))
    else:
        prepared = S.protein_queries(inputs.query_sequences)
    chunks = database_chunks(inputs, chunk_counts)
    e = N.PresearchEngine(0)
    try:
        if graph:
            e.set_graph(True)
        rows = S.search(e, p, prepared, chunks,
                        N.SCHEDULE_BATCHED if schedule is None else schedule)
    finally:
        e.close()
    return S.hit_table(rows, prepared, chunks, inputs.query_names, inputs.subject_names)
