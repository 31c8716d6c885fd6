"""The reference's own programs timed and checked on slices of a benchmark
workload (test infrastructure: the benchmark's reference arm, its CPU
baseline and its parity check; never the engine).

The reference's CPU search (`ghostz aln -g 0 -a <threads>`, oracle/_ref/ghostz
compiled from the reference's sources) runs on two database slices, the
first S1 and the first S2 sequences of the workload's database, each built
by the reference's `ghostz db` beforehand (untimed, as `db` is a separate
step).  Its time is taken as t(R) = a + b R over the slices' residues R (a:
per-query work that does not depend on the database -- reading, SEG,
statistics, query lists; b: the search), and the whole database's time is
read off that line: t_full = t1 + (t2 - t1) (R_full - R1) / (R2 - R1).
The slices are the first 40,000 and 160,000 sequences: the search's time
per residue falls as the database grows, so a line through smaller slices
(20,000 and 40,000) over-estimated the whole database's time, and its
short difference t2 - t1 made the estimate noisy.

The parity check runs the reference's GPU aligner (`ghostz-gpu aln -g 1`,
its host code on CPU stand-in operators) on the first slice.
"""
from __future__ import annotations

import os
import shutil
import tempfile
import time

import numpy as np

import ref_aln as R

PROTEIN_LETTERS = np.frombuffer(b"ARNDCQEGHILKMFPSTWYVBJZ*X", np.uint8)


def _letters(codes):
    return PROTEIN_LETTERS[np.asarray(codes, np.int64)].tobytes()


class ReferenceSlices:
    """A workload's queries and slices of its database (two for timing, one
    for the parity check), written as the reference's FASTA inputs and
    databases under a scratch directory."""

    def __init__(self, db, query_sequences, slices=(40_000, 160_000), threads=None,
                 clustering=True):
        self.dir = tempfile.mkdtemp(prefix="gz_ref_")
        self.threads = threads or os.cpu_count() or 1
        self.n_queries = len(query_sequences)
        self.slices = [min(s, db.number_sequences) for s in slices]
        self.full_residues = int(db.length) - db.number_sequences - 1
        self.query_fasta = os.path.join(self.dir, "q.fa")
        R.write_fasta(self.query_fasta, [f"q{i}" for i in range(self.n_queries)],
                      [_letters(s) for s in query_sequences])
        self.prefixes, self.residues = [], []
        t = time.perf_counter()
        for n in self.slices:
            fa = os.path.join(self.dir, f"db{n}.fa")
            R.write_fasta(fa, [f"s{j}" for j in range(n)],
                          [_letters(db.codes[int(db.offsets[j]):int(db.offsets[j + 1]) - 1])
                           for j in range(n)])
            prefix = os.path.join(self.dir, f"db{n}")
            R.build_database(fa, prefix, clustering=clustering, threads=self.threads)
            self.prefixes.append(prefix)
            self.residues.append(int(db.offsets[n]) - n - 1)
        self.db_build_s = time.perf_counter() - t

    def close(self):
        shutil.rmtree(self.dir, ignore_errors=True)

    def time_slices(self):
        """One `ghostz aln -g 0 -a threads` of all queries on each slice:
        (seconds on slice 1, seconds on slice 2)."""
        out = os.path.join(self.dir, "out.txt")
        return tuple(R.align(self.query_fasta, p, out, threads=self.threads)
                     for p in self.prefixes)

    def full_seconds(self, t1, t2):
        """The whole database's time on the line through the two slices; a
        slope no larger than zero (timing noise) falls back to scaling the
        larger slice's time by the residue ratio."""
        r1, r2 = self.residues
        if r2 > r1 and t2 > t1:
            return t1 + (t2 - t1) * (self.full_residues - r1) / (r2 - r1)
        return t2 * self.full_residues / r2

    def describe(self, t1, t2):
        s1, s2 = self.slices
        return (f"reference `ghostz aln -g 0 -a {self.threads}` (compiled from the reference's "
                f"sources): {self.n_queries} queries x first {s1} and first {s2} DB sequences "
                f"({self.residues[0]} and {self.residues[1]} residues) in {t1:.2f} s and "
                f"{t2:.2f} s; the whole database's {self.full_residues} residues read off the "
                f"line through both (queries' own work counted once)")

    def gpu_aligner_table(self, n_queries):
        """The reference GPU aligner's hit table of the first n_queries
        queries against the first slice."""
        q = os.path.join(self.dir, f"q{n_queries}.fa")
        with open(self.query_fasta, "rb") as f:
            records = f.read().split(b">")[1:n_queries + 1]
        with open(q, "wb") as f:
            f.write(b"".join(b">" + r for r in records))
        out = os.path.join(self.dir, "parity.txt")
        R.align(q, self.prefixes[0], out, threads=self.threads, gpu_aligner=True)
        return R.read_table(out)
