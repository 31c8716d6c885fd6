"""One `aln` search on the GPU, from query residues to the tabular hit lines.

The steps of the reference's GPU search for one query set
(AlignerGpu::Align / Presearch / BuildResults, src/aligner_gpu.cpp:44-340):

1. query preparation: protein queries are SEG-masked (`-F T`) or six-frame
   translated reads are translated and masked, and every query gets its
   ungapped X-drop and gapped trigger (src/aligner_gpu.cpp:213-242) --
   on the GPU (`prepare_protein_queries`, `prepare_translated_queries`);
2. the presearch of every database chunk in chunk order, merged per query
   into the top-b lists (AlignerGpuPresearchThread's chunk loop,
   src/aligner_gpu_presearch_thread.cpp:214-640) -- `gzb_engine_presearch`;
3. the build results step chunk by chunk (AlignerBuildResultsThread::Run,
   src/aligner_build_results_thread.h:64-178) -- `gzb_engine_build_alignments`;
4. each query's results in the reference's final order (:179-190) --
   `gzb_sort_alignments`;
5. the tabular lines (AlignerCommon::WriteOutput,
   src/aligner_common.h:344-394) -- `gzb_write_hit_table`.

Chunks are stored on the device after their presearch (`swap_database`),
so the build step needs no second index build.  File reading and writing
stay with the caller: inputs are residue codes and names.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import native as N
from . import params as P
from . import workload as W


@dataclass
class PreparedQueries:
    queries: W.Queries            # engine layout, masked codes, cutoffs
    real_lengths: np.ndarray      # residues (a read's bases // 3 translated)
    dna_lengths: Optional[np.ndarray] = None  # bases per read, translated only


def protein_queries(letters: Sequence[bytes], filter: bool = True) -> PreparedQueries:
    """Protein queries given as letters (what a FASTA record holds): SEG
    (when `filter`) and cutoffs on the GPU (ProteinQuery,
    src/protein_query.cpp:39-49)."""
    # lower-case letters carry code + 32 so SEG leaves them out of its
    # compositions; without the filter they are plain residues
    seqs = [N.encode_protein_for_seg(s) for s in letters]
    if not filter:
        seqs = [s & 31 for s in seqs]
    q = W.pack_queries([s & 31 for s in seqs],
                       cutoffs=(np.zeros(len(seqs), np.int32), np.zeros(len(seqs), np.int32)))
    raw = q.codes.copy()
    for i, s in enumerate(seqs):
        o = int(q.offsets[i])
        raw[o + 1:o + 1 + len(s)] = s
    codes, cut, trig = N.prepare_protein_queries(raw, q.offsets, q.lengths, filter=filter)
    q.codes, q.cutoffs, q.triggers = codes, cut, trig
    real = q.lengths.astype(np.int64) - 2
    return PreparedQueries(queries=q, real_lengths=real.astype(np.uint32))


def translated_queries(dna: np.ndarray, offsets: np.ndarray,
                       filter: bool = True) -> PreparedQueries:
    """DNA reads (ASCII bases back to back, number_reads + 1 boundaries):
    six-frame translation, SEG and cutoffs on the GPU (TranslatedDnaQuery,
    src/translated_dna_query.cpp:44-85); the real length of a read's query
    is its bases // 3 (src/translated_dna_query.h)."""
    codes, offs, lens, cut, trig = N.prepare_translated_queries(dna, offsets, filter=filter)
    q = W.translated_queries(codes, offs, lens, cutoffs=(cut, trig))
    dna_lengths = np.diff(np.asarray(offsets, dtype=np.int64)).astype(np.uint32)
    return PreparedQueries(queries=q, real_lengths=(dna_lengths // 3).astype(np.uint32),
                           dna_lengths=dna_lengths)


def search(engine: "N.PresearchEngine", params, prepared: PreparedQueries,
           chunks: List[W.Database], schedule: int = N.SCHEDULE_BATCHED):
    """Steps 2-4 for the prepared queries over the database `chunks` (chunk
    k gets chunk id k): returns, per query, its alignment records in the
    order the reference writes them, with subject ids counted over all
    chunks (chunk k's subjects follow those of chunks 0..k-1)."""
    engine.set_params(params)
    engine.set_queries(prepared.queries)
    engine.reset_results()
    for k, db in enumerate(chunks):
        engine.set_database(db, chunk_id=k)
        engine.presearch(schedule)
        if len(chunks) > 1:
            engine.swap_database(k)  # stored in slot k, resident slot empty
    merged = engine.results()
    rows = [np.zeros(len(r), N.ALIGNMENT_DTYPE) for r in merged]
    base = np.concatenate([[0], np.cumsum([db.number_sequences for db in chunks])])
    for k in range(len(chunks)):
        if len(chunks) > 1:
            engine.swap_database(k)
        built = engine.build_alignments()
        if len(chunks) > 1:
            engine.swap_database(k)
        for qi, b in enumerate(built):
            mine = b["chunk_id"] == k
            rows[qi][mine] = b[mine]
            rows[qi]["subject_id"][mine] += int(base[k])
    offsets = global_offsets(chunks)
    return N.sort_alignments(rows, offsets, int(base[-1]), prepared.dna_lengths)


def global_offsets(chunks: List[W.Database]) -> np.ndarray:
    """First-residue offsets of every subject, each within its own chunk,
    indexed by the subject ids search() returns."""
    if not chunks:
        return np.zeros(1, np.uint32)
    return np.concatenate([db.offsets[:-1] for db in chunks] + [np.zeros(1, np.uint32)]) \
        .astype(np.uint32)


def hit_table(rows, prepared: PreparedQueries, chunks: List[W.Database],
              query_names: Sequence[str], subject_names: Sequence[str]) -> List[str]:
    """Step 5: the `aln` lines of search()'s records.  subject_names are
    those of all chunks in chunk order; the search space counts residues
    and sequences of the whole database (Database::GetDatabaseTotalLenght /
    GetNumberTotalSequences)."""
    db_length = sum(int(db.length) - db.number_sequences - 1 for db in chunks)
    db_sequences = sum(db.number_sequences for db in chunks)
    return N.hit_table(rows, list(query_names), list(subject_names), global_offsets(chunks),
                       db_length, db_sequences, prepared.real_lengths,
                       dna_lengths=prepared.dna_lengths)
