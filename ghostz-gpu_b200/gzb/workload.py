"""Seeded synthetic protein workloads with the shapes of the benchmark
configurations: log-normal lengths, i.i.d. residues from the Robinson
background, and planted homologs mutated by BLOSUM62-conditional
substitution to 30-90 % identity with geometric indels.

A database is the reference's concatenated chunk layout
``[delim s0 delim s1 ... delim]`` with ``offsets[i]`` = first residue of
sequence i (src/database_chunk.h:282-300).  Queries use the protein-query
framing ``[delim residues delim]`` (src/protein_query.cpp:39-49) and are
concatenated sharing delimiters, ``offsets[i]`` = leading delimiter of query
i (src/aligner_gpu.cpp:213-242).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import params as P


@dataclass
class Database:
    codes: np.ndarray            # uint8, concatenated with delimiters
    offsets: np.ndarray          # uint32, number_sequences + 1
    number_sequences: int

    @property
    def length(self) -> int:
        return int(self.codes.shape[0])


@dataclass
class Queries:
    codes: np.ndarray            # uint8, concatenated, shared delimiters
    offsets: np.ndarray          # uint32, leading delimiter of each query
    lengths: np.ndarray          # uint32, residues + 2
    cutoffs: np.ndarray          # int32 ungapped X-drop per query
    triggers: np.ndarray         # int32 gapped-extension trigger per query
    sources: np.ndarray = field(default=None)  # planted homolog source or -1

    @property
    def number(self) -> int:
        return int(self.offsets.shape[0])


def _background_probs():
    f = np.zeros(len(P.REGULAR))
    for ch, v in P.ROBINSON.items():
        f[P.REGULAR.index(ch)] = v
    return f / f.sum()


def lognormal_lengths(rng, n, median, sigma, lo, hi):
    x = rng.lognormal(mean=np.log(median), sigma=sigma, size=n)
    return np.clip(np.rint(x), lo, hi).astype(np.int64)


def random_residues(rng, n, chunk=1 << 26):
    """n i.i.d. residue codes from the background, as uint8 (chunked inverse
    CDF on 32-bit uniforms, so large draws need no 64-bit temporaries)."""
    cdf = np.cumsum(_background_probs())
    thresholds = np.minimum(np.round(cdf * 2.0**32), 2.0**32 - 1).astype(np.uint64)[:-1]
    out = np.empty(n, dtype=np.uint8)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        u = rng.integers(0, 2**32, size=b - a, dtype=np.uint64)
        out[a:b] = np.searchsorted(thresholds, u, side="right").astype(np.uint8)
    return out


def make_database(n_sequences, seed, median=300, sigma=0.6, lo=30, hi=3000):
    rng = np.random.default_rng(seed)
    lens = lognormal_lengths(rng, n_sequences, median, sigma, lo, hi)
    total = int(lens.sum()) + n_sequences + 1
    offsets = np.empty(n_sequences + 1, dtype=np.uint32)
    starts = np.concatenate([[1], 1 + np.cumsum(lens + 1)[:-1]]).astype(np.int64)
    offsets[:-1] = starts
    offsets[-1] = total
    codes = random_residues(rng, total)
    codes[0] = P.DELIMITER
    codes[starts + lens] = P.DELIMITER  # delimiter after every sequence
    return Database(codes=codes, offsets=offsets, number_sequences=n_sequences)


def _substitution_table(lam=0.3176):
    m = P.blosum62()[:20, :20].astype(np.float64)
    bg = _background_probs()
    t = bg[None, :] * np.exp(lam * m)
    np.fill_diagonal(t, 0.0)
    return t / t.sum(axis=1, keepdims=True)


def mutate(rng, seq, identity, indel_p=0.02, indel_mean=3.0):
    """BLOSUM62-conditional substitutions at rate 1-identity, plus
    insertions/deletions at indel_p per site with geometric lengths."""
    table = np.cumsum(_substitution_table(), axis=1)
    seq = np.asarray(seq, dtype=np.uint8).copy()
    sub = np.nonzero(rng.random(len(seq)) < (1.0 - identity))[0]
    if len(sub):
        u = rng.random(len(sub))
        rows = table[seq[sub]]
        seq[sub] = np.minimum((rows < u[:, None]).sum(axis=1), 19).astype(np.uint8)
    events = np.nonzero(rng.random(len(seq)) < indel_p)[0]
    if len(events) == 0:
        return seq
    pieces = []
    prev = 0
    for i in events:
        if i < prev:
            continue
        pieces.append(seq[prev:i])
        k = int(rng.geometric(1.0 / indel_mean))
        if rng.random() < 0.5:
            pieces.append(random_residues(rng, k))
            prev = i
        else:
            prev = i + k
    pieces.append(seq[prev:])
    out = np.concatenate(pieces)
    return out if len(out) else seq[:1]


def make_queries(db: Database, n_queries, seed, homolog_fraction=0.3,
                 median=300, sigma=0.6, lo=30, hi=3000, cutoffs=None):
    rng = np.random.default_rng(seed)
    lens = lognormal_lengths(rng, n_queries, median, sigma, lo, hi)
    seqs = []
    sources = np.full(n_queries, -1, dtype=np.int64)
    for i in range(n_queries):
        if rng.random() < homolog_fraction:
            s = int(rng.integers(db.number_sequences))
            a, b = int(db.offsets[s]), int(db.offsets[s + 1]) - 1
            src = db.codes[a:b]
            ident = rng.uniform(0.3, 0.9)
            seqs.append(mutate(rng, src, ident))
            sources[i] = s
        else:
            seqs.append(random_residues(rng, int(lens[i])))
    return pack_queries(seqs, sources=sources, cutoffs=cutoffs)


def pack_queries(seqs, sources=None, cutoffs=None) -> Queries:
    n = len(seqs)
    lengths = np.array([len(s) + 2 for s in seqs], dtype=np.uint32)
    total = int((lengths - 1).sum()) + 1
    codes = np.empty(total, dtype=np.uint8)
    offsets = np.empty(n, dtype=np.uint32)
    off = 0
    for i, s in enumerate(seqs):
        offsets[i] = off
        codes[off] = P.DELIMITER
        codes[off + 1: off + 1 + len(s)] = s
        off += len(s) + 1
    codes[off] = P.DELIMITER
    if cutoffs is None:
        cut, trig = P.query_cutoffs(seqs)
    else:
        cut, trig = cutoffs
    return Queries(codes=codes, offsets=offsets, lengths=lengths, cutoffs=cut,
                   triggers=trig,
                   sources=sources if sources is not None else np.full(n, -1))


def query_sequences(q: Queries):
    """Residue arrays (no delimiters) of every query."""
    return [q.codes[int(o) + 1:int(o) + int(l) - 1] for o, l in zip(q.offsets, q.lengths)]


# -- translated-DNA workload ----------------------------------------------------
# the standard genetic code, codons in ACGT order (first base slowest)
_CODON_LETTERS = "KNKNTTTTRSRSIIMIQHQHPPPPRRRRLLLLEDEDAAAAGGGGVVVV*Y*YSSSS*CWCLFLF"
_BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
_COMPLEMENT = np.zeros(256, dtype=np.uint8)
for _a, _b in zip(b"ACGT", b"TGCA"):
    _COMPLEMENT[_a] = _b


@dataclass
class Reads:
    dna: np.ndarray              # uint8 ASCII bases of all reads back to back
    offsets: np.ndarray          # uint64, number_reads + 1 boundaries
    sources: np.ndarray = field(default=None)  # planted fragment source or -1

    @property
    def number(self) -> int:
        return int(self.offsets.shape[0]) - 1

    def read(self, i) -> bytes:
        return self.dna[int(self.offsets[i]):int(self.offsets[i + 1])].tobytes()


def _codon_choices():
    """(20, 6) codon indices per regular residue code and their counts."""
    table = np.zeros((len(P.REGULAR), 6), dtype=np.int64)
    count = np.zeros(len(P.REGULAR), dtype=np.int64)
    for c, letter in enumerate(_CODON_LETTERS):
        if letter in P.REGULAR:
            a = P.REGULAR.index(letter)
            table[a, count[a]] = c
            count[a] += 1
    return table, count


def make_reads(db: Database, n_reads, seed, read_length=150, homolog_fraction=0.4,
               error=0.01) -> Reads:
    """Synthetic reads of one length with i.i.d. bases at 50 % GC; a
    fraction are reverse-translated fragments of random database proteins
    (uniform codon choice, random strand and frame) with per-base
    substitution errors."""
    rng = np.random.default_rng(seed)
    reads = _BASES[rng.integers(0, 4, size=(n_reads, read_length))]
    planted = rng.random(n_reads) < homolog_fraction
    sources = np.full(n_reads, -1, dtype=np.int64)
    idx = np.flatnonzero(planted)
    if len(idx):
        k = read_length // 3 + 1  # residues covering every frame offset
        s = rng.integers(0, db.number_sequences, size=len(idx))
        first = db.offsets[s].astype(np.int64)
        plen = db.offsets[s + 1].astype(np.int64) - 1 - first
        start = (rng.random(len(idx)) * np.maximum(plen - k + 1, 1)).astype(np.int64)
        pos = start[:, None] + np.arange(k)[None, :]
        inside = pos < plen[:, None]
        res = db.codes[np.minimum(first[:, None] + pos, db.length - 1)].astype(np.int64)
        res = np.where(inside & (res < len(P.REGULAR)), res,
                       rng.integers(0, len(P.REGULAR), size=res.shape))
        table, count = _codon_choices()
        pick = (rng.random(res.shape) * count[res]).astype(np.int64)
        codon = table[res, pick]                      # (m, k) codon indices
        nt = np.stack([codon // 16, (codon // 4) % 4, codon % 4], axis=-1).reshape(len(idx), -1)
        frame = rng.integers(0, 3, size=len(idx))
        nt = np.take_along_axis(nt, frame[:, None] + np.arange(read_length)[None, :], axis=1)
        frag = _BASES[nt]
        rev = rng.random(len(idx)) < 0.5
        frag[rev] = _COMPLEMENT[frag[rev][:, ::-1]]
        hit = rng.random(frag.shape) < error
        shift = rng.integers(1, 4, size=frag.shape)
        code = np.searchsorted(_BASES, frag)
        frag = np.where(hit, _BASES[(code + shift) % 4], frag)
        reads[idx] = frag
        sources[idx] = s
    offsets = np.arange(n_reads + 1, dtype=np.uint64) * np.uint64(read_length)
    return Reads(dna=reads.reshape(-1).copy(), offsets=offsets, sources=sources)


def translated_queries(codes, offsets, lengths, sources=None, cutoffs=None) -> Queries:
    """Queries over translated reads already laid out with shared
    delimiters (the output of six-frame translation): per-query cutoffs
    from each translated query's own composition, as
    TranslatedDnaQuery::SetStaticalParameters does
    (src/translated_dna_query.cpp:76-85)."""
    offsets = np.asarray(offsets, dtype=np.uint32)
    lengths = np.asarray(lengths, dtype=np.uint32)
    if cutoffs is None:
        seqs = [codes[int(o) + 1:int(o) + int(n) - 1] for o, n in zip(offsets, lengths)]
        cutoffs = P.query_cutoffs(seqs)
    cut, trig = cutoffs
    n = len(offsets)
    return Queries(codes=np.asarray(codes, dtype=np.uint8), offsets=offsets, lengths=lengths,
                   cutoffs=cut, triggers=trig,
                   sources=sources if sources is not None else np.full(n, -1))
