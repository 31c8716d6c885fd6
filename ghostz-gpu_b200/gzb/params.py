"""Search parameters for the presearch engine: alphabet coding, BLOSUM62,
reduced alphabets, seed-hash code scores and nominal cutoffs.

Everything here is host-side set-up that the reference computes before it
calls its GPU operators; the engine receives the results as plain arrays.

* Alphabet: protein letters ``ARNDCQEGHILKMFPSTWYV`` (codes 0-19), ambiguous
  ``BJZ*`` (20-23), unknown ``X`` (24), delimiter 25
  (src/protein_type.cpp:12-14, src/alphabet_coder.cpp:25-50,
  src/aligner_common.cpp:70-73).
* Reduced alphabet ``A KR EDNQ C G H ILVM FYW P ST``: each letter maps to the
  first letter of its set; codes are handed out in alphabet order to set
  representatives, then to ambiguous and unknown letters
  (src/reduced_alphabet_coder.cpp:30-98, src/database_build_main.cpp:60-62).
* Code scores: per reduced code the largest self score of its letters
  (src/seed_searcher_database_parameters.cpp:55-64).
* Thresholds use float arithmetic as the reference does
  (src/seed_searcher_gpu.cpp:64-67,
  src/seed_searcher_database_parameters.cpp:409-411,
  src/statistics.cpp:28-43).
"""
from __future__ import annotations

import math

import numpy as np

REGULAR = "ARNDCQEGHILKMFPSTWYV"
AMBIGUOUS = "BJZ*"
UNKNOWN = "X"
LETTERS = REGULAR + AMBIGUOUS + UNKNOWN  # code = index
NUMBER_LETTERS = len(LETTERS)  # 25
DELIMITER = NUMBER_LETTERS  # 25
DEFAULT_REDUCED_SETS = "A KR EDNQ C G H ILVM FYW P ST"

# BLOSUM62 (Henikoff & Henikoff 1992), the standard published matrix, in the
# row/column order below; J is absent from the published table and scores 0.
_B62_ORDER = "ARNDCQEGHILKMFPSTWYVBZX*"
_B62_ROWS = [
    [4, -1, -2, -2, 0, -1, -1, 0, -2, -1, -1, -1, -1, -2, -1, 1, 0, -3, -2, 0, -2, -1, 0, -4],
    [-1, 5, 0, -2, -3, 1, 0, -2, 0, -3, -2, 2, -1, -3, -2, -1, -1, -3, -2, -3, -1, 0, -1, -4],
    [-2, 0, 6, 1, -3, 0, 0, 0, 1, -3, -3, 0, -2, -3, -2, 1, 0, -4, -2, -3, 3, 0, -1, -4],
    [-2, -2, 1, 6, -3, 0, 2, -1, -1, -3, -4, -1, -3, -3, -1, 0, -1, -4, -3, -3, 4, 1, -1, -4],
    [0, -3, -3, -3, 9, -3, -4, -3, -3, -1, -1, -3, -1, -2, -3, -1, -1, -2, -2, -1, -3, -3, -2, -4],
    [-1, 1, 0, 0, -3, 5, 2, -2, 0, -3, -2, 1, 0, -3, -1, 0, -1, -2, -1, -2, 0, 3, -1, -4],
    [-1, 0, 0, 2, -4, 2, 5, -2, 0, -3, -3, 1, -2, -3, -1, 0, -1, -3, -2, -2, 1, 4, -1, -4],
    [0, -2, 0, -1, -3, -2, -2, 6, -2, -4, -4, -2, -3, -3, -2, 0, -2, -2, -3, -3, -1, -2, -1, -4],
    [-2, 0, 1, -1, -3, 0, 0, -2, 8, -3, -3, -1, -2, -1, -2, -1, -2, -2, 2, -3, 0, 0, -1, -4],
    [-1, -3, -3, -3, -1, -3, -3, -4, -3, 4, 2, -3, 1, 0, -3, -2, -1, -3, -1, 3, -3, -3, -1, -4],
    [-1, -2, -3, -4, -1, -2, -3, -4, -3, 2, 4, -2, 2, 0, -3, -2, -1, -2, -1, 1, -4, -3, -1, -4],
    [-1, 2, 0, -1, -3, 1, 1, -2, -1, -3, -2, 5, -1, -3, -1, 0, -1, -3, -2, -2, 0, 1, -1, -4],
    [-1, -1, -2, -3, -1, 0, -2, -3, -2, 1, 2, -1, 5, 0, -2, -1, -1, -1, -1, 1, -3, -1, -1, -4],
    [-2, -3, -3, -3, -2, -3, -3, -3, -1, 0, 0, -3, 0, 6, -4, -2, -2, 1, 3, -1, -3, -3, -1, -4],
    [-1, -2, -2, -1, -3, -1, -1, -2, -2, -3, -3, -1, -2, -4, 7, -1, -1, -4, -3, -2, -2, -1, -2, -4],
    [1, -1, 1, 0, -1, 0, 0, 0, -1, -2, -2, 0, -1, -2, -1, 4, 1, -3, -2, -2, 0, 0, 0, -4],
    [0, -1, 0, -1, -1, -1, -1, -2, -2, -1, -1, -1, -1, -2, -1, 1, 5, -2, -2, 0, -1, -1, 0, -4],
    [-3, -3, -4, -4, -2, -2, -3, -2, -2, -3, -2, -3, -1, 1, -4, -3, -2, 11, 2, -3, -4, -3, -2, -4],
    [-2, -2, -2, -3, -2, -1, -2, -3, 2, -1, -1, -2, -1, 3, -3, -2, -2, 2, 7, -1, -3, -2, -1, -4],
    [0, -3, -3, -3, -1, -2, -2, -3, -3, 3, 1, -2, 1, -1, -2, -2, 0, -3, -1, 4, -3, -2, -1, -4],
    [-2, -1, 3, 4, -3, 0, 1, -1, 0, -3, -4, 0, -3, -3, -2, 0, -1, -4, -3, -3, 4, 1, -1, -4],
    [-1, 0, 0, 1, -3, 3, 4, -2, 0, -3, -3, 1, -1, -3, -1, 0, -1, -3, -2, -2, 1, 4, -1, -4],
    [0, -1, -1, -1, -2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -2, 0, 0, -2, -1, -1, -1, -1, -1, -4],
    [-4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, -4, 1],
]

# Background amino-acid frequencies of Robinson & Robinson (1991), the table
# the reference uses for ungapped Karlin statistics (src/statistics.cpp:154-175).
ROBINSON = {
    "L": 90.19, "A": 78.05, "G": 73.77, "S": 71.20, "V": 64.41, "E": 62.95,
    "T": 58.41, "K": 57.44, "D": 53.64, "P": 52.03, "I": 51.42, "R": 51.29,
    "N": 44.87, "Q": 42.64, "F": 38.56, "Y": 32.16, "M": 22.43, "H": 21.99,
    "C": 19.25, "W": 13.30,
}

GAPPED_LAMBDA = 0.267  # BLOSUM62 11/1 (src/statistics.cpp:236-240)
GAPPED_K = 0.041


def encode(text: str) -> np.ndarray:
    """Letters -> residue codes; anything unknown becomes X (24)."""
    table = np.full(256, LETTERS.index(UNKNOWN), dtype=np.uint8)
    for i, ch in enumerate(LETTERS):
        table[ord(ch)] = i
        table[ord(ch.lower())] = i
    return table[np.frombuffer(text.encode("ascii"), dtype=np.uint8)]


def blosum62() -> np.ndarray:
    """25x25 int32 matrix in code order ([row code, column code])."""
    m = np.zeros((NUMBER_LETTERS, NUMBER_LETTERS), dtype=np.int32)
    for i, a in enumerate(_B62_ORDER):
        for j, b in enumerate(_B62_ORDER):
            m[LETTERS.index(a), LETTERS.index(b)] = _B62_ROWS[i][j]
    return m


def reduced_code_map(sets: str = DEFAULT_REDUCED_SETS):
    """Residue code -> reduced code, and the largest regular reduced code."""
    groups = sets.split()

    def rep(ch):
        for g in groups:
            if ch in g:
                return g[0]
        return ch

    code_of = {}
    nxt = 0
    regular_count = 0
    for ch in REGULAR:
        if rep(ch) == ch:
            regular_count += 1
    for ch in LETTERS:
        if rep(ch) == ch:
            code_of[ch] = nxt
            nxt += 1
    out = np.zeros(NUMBER_LETTERS, dtype=np.uint8)
    for i, ch in enumerate(LETTERS):
        out[i] = code_of[rep(ch)]
    return out, regular_count - 1


PARAMS_DTYPE = np.dtype([
    ("delimiter", "<i4"),
    ("number_letters", "<i4"),
    ("score_matrix", "<i4", (32 * 32,)),
    ("map_size", "<i4"),
    ("hash_code_map", "u1", (32,)),
    ("similarity_code_map", "u1", (32,)),
    ("max_indexing_code", "<i4"),
    ("code_scores", "<i4", (32,)),
    ("seed_threshold", "<i4"),
    ("max_hash_length", "<i4"),
    ("min_hash_length", "<i4"),
    ("subsequence_length", "<i4"),
    ("max_member_distance", "<i4"),
    ("distance_threshold", "<i4"),
    ("gap_open", "<i4"),
    ("gap_extension", "<i4"),
    ("gapped_cutoff", "<i4"),
    ("max_number_results", "<i4"),
    ("max_number_one_subject_results", "<i4"),
    ("clustering", "<i4"),
    ("result_gapped_cutoff", "<i4"),
], align=False)


def normalized_to_nominal(bits: float, lam: float, k: float) -> int:
    """floor((bits*ln2 + ln K)/lambda) in float32 (src/statistics.cpp:33-37)."""
    f = np.float32
    v = (f(bits) * f(math.log(2.0)) + np.log(f(k))) / f(lam)
    return int(np.floor(f(v)))


def normalized_cutoff_to_nominal(bits: float, lam: float) -> int:
    """floor(bits*ln2/lambda) in float32 (src/statistics.cpp:39-43)."""
    f = np.float32
    v = (f(bits) * f(math.log(2.0))) / f(lam)
    return int(np.floor(f(v)))


def make_params(*, subsequence_length=10, seed_threshold=39, gap_open=11,
                gap_extension=1, gapped_bits=15.0, max_number_results=10,
                max_number_one_subject_results=1, clustering=True,
                matrix=None, reduced_sets=DEFAULT_REDUCED_SETS,
                gapped_cutoff=None, result_gapped_bits=25.0,
                result_gapped_cutoff=None) -> np.ndarray:
    """One record of PARAMS_DTYPE with the `aln` defaults
    (src/align_main.cpp:104-127, src/database_build_main.cpp:72-81)."""
    p = np.zeros(1, dtype=PARAMS_DTYPE)[0]
    m = blosum62() if matrix is None else np.asarray(matrix, dtype=np.int32)
    n = m.shape[0]
    p["delimiter"] = DELIMITER
    p["number_letters"] = n
    sm = np.zeros(32 * 32, dtype=np.int32)
    sm[: n * n] = m.reshape(-1)
    p["score_matrix"] = sm
    p["map_size"] = n
    rmap, max_regular = reduced_code_map(reduced_sets)
    hm = np.zeros(32, dtype=np.uint8)
    hm[:n] = rmap[:n]
    p["hash_code_map"] = hm
    p["similarity_code_map"] = hm
    p["max_indexing_code"] = max_regular
    cs = np.zeros(32, dtype=np.int32)
    for i in range(n):
        c = int(rmap[i])
        if c <= max_regular:
            cs[c] = max(cs[c], int(m[i, i]))
    p["code_scores"] = cs
    p["seed_threshold"] = seed_threshold
    p["max_hash_length"] = 8
    p["min_hash_length"] = 6
    L = subsequence_length
    f = np.float32
    p["subsequence_length"] = L
    p["max_member_distance"] = int(f(L) * (f(1.0) - f(0.9)))
    p["distance_threshold"] = int(f(L) - f(0.8) * f(L))
    p["gap_open"] = gap_open
    p["gap_extension"] = gap_extension
    if gapped_cutoff is None:
        gapped_cutoff = normalized_to_nominal(gapped_bits, GAPPED_LAMBDA, GAPPED_K)
    p["gapped_cutoff"] = gapped_cutoff
    p["max_number_results"] = max_number_results
    p["max_number_one_subject_results"] = max_number_one_subject_results
    p["clustering"] = 1 if clustering else 0
    # the build results step re-extends with a wider X-drop than the
    # presearch (normalized_result_gapped_extension_cutoff, 25 bits)
    if result_gapped_cutoff is None:
        result_gapped_cutoff = normalized_to_nominal(result_gapped_bits, GAPPED_LAMBDA, GAPPED_K)
    p["result_gapped_cutoff"] = result_gapped_cutoff
    return p


# ---------------------------------------------------------------------------
# Ungapped Karlin-Altschul parameters of one query against the background
# (the statistics the reference takes per query in
# src/statistics.cpp:205-229 via ext/karlin/src/karlin.c).
# lambda solves sum_s p_s exp(lambda s) = 1 (Newton, stopped at 1e-5
# relative change); H = lambda sum_s s p_s exp(lambda s); K follows Karlin &
# Altschul (1990) for scores of span delta:
#   K = delta exp(-2 sigma) / ((H/lambda) (1 - exp(-lambda delta))),
#   sigma = sum_k (1/k) [E(exp(lambda S_k); S_k < 0) + P(S_k >= 0)],
# with the series summed while its terms exceed 0.01 and then closed with a
# geometric tail down to 1e-4, lambda and H rounded to float first, as the
# reference's statistics library does.
def _score_probabilities(matrix, f1, f2):
    lo, hi = int(matrix.min()), int(matrix.max())
    w = (np.asarray(f1)[:, None] * np.asarray(f2)[None, :]).reshape(-1)
    probs = np.bincount((matrix.reshape(-1) - lo), weights=w, minlength=hi - lo + 1)
    s = probs[probs > 0].sum()
    probs = np.where(probs > 0, probs / s, 0.0)
    return probs, lo, hi


def karlin(probs, lo, hi):
    scores = np.arange(lo, hi + 1, dtype=np.float64)
    mean = float((scores * probs).sum())
    if mean >= 0 or hi <= 0:
        raise ValueError("expected score must be negative and a positive score must exist")
    lam = 0.5
    for _ in range(20):
        e = probs * np.exp(lam * scores)
        step = (e.sum() - 1.0) / float((scores * e).sum())
        lam -= step
        if abs(step / lam) < 1e-5:
            e = probs * np.exp(lam * scores)
            lam -= (e.sum() - 1.0) / float((scores * e).sum())
            break
    lam = float(np.float32(lam))
    H = float(np.float32(lam * float((scores * probs * np.exp(lam * scores)).sum())))
    if lo == -1 or hi == 1:
        return lam, float(np.float32(H / lam * (1.0 - math.exp(-lam)))), H
    sumlimit = 0.01
    total = 0.0
    term = 1.0
    old, old2 = 1.0, 1.0
    dist = np.array([1.0])
    off = 0
    j = 0
    while j < 100 and term > sumlimit:
        dist = np.convolve(dist, probs)
        off += lo
        s = np.arange(off, off + len(dist), dtype=np.float64)
        neg = s < 0
        inner = float((dist[neg] * np.exp(lam * s[neg])).sum() + dist[~neg].sum())
        old2, old = old, inner
        j += 1
        term = inner / j
        total += term
    ratio = old / old2
    if ratio >= 1.0 - sumlimit * 0.001:
        return lam, -1.0, H
    sumlimit *= 0.01
    while term > sumlimit:
        old *= ratio
        j += 1
        term = old / j
        total += term
    delta = 0
    for i in range(1, hi - lo + 1):
        if probs[i] > 0:
            delta = i if delta == 0 else math.gcd(delta, i)
    delta = math.gcd(delta, -lo) if delta else -lo
    av = H / lam
    K = delta * math.exp(-2.0 * total) / (av * (1.0 - math.exp(-lam * delta)))
    return lam, float(np.float32(K)), H


def _background():
    f = np.zeros(NUMBER_LETTERS)
    for ch, v in ROBINSON.items():
        f[LETTERS.index(ch)] = v
    return f / f.sum()


def ungapped_karlin_for_query(codes: np.ndarray, matrix=None):
    """(lambda, K, H) of one query (codes without delimiters).  Frequencies
    count regular letters plus one pseudo-count for any letter seen less
    than once (src/statistics.cpp:328-347)."""
    m = blosum62() if matrix is None else matrix
    freq = np.zeros(NUMBER_LETTERS)
    c = codes[codes < len(REGULAR)]
    if len(c):
        freq[: len(REGULAR)] = np.bincount(c, minlength=len(REGULAR))[: len(REGULAR)]
    freq[freq < 1.0] += 1.0
    freq /= freq.sum()
    probs, lo, hi = _score_probabilities(m, freq, _background())
    return karlin(probs, lo, hi)


def query_cutoffs(query_codes_list, ungapped_bits=7.0, trigger_bits=22.0,
                  matrix=None):
    """Per-query ungapped X-drop and gapped-extension trigger
    (src/aligner_gpu.cpp:213-242)."""
    cut = np.zeros(len(query_codes_list), dtype=np.int32)
    trig = np.zeros(len(query_codes_list), dtype=np.int32)
    cache = {}
    for i, q in enumerate(query_codes_list):
        comp = np.bincount(q[q < len(REGULAR)], minlength=len(REGULAR)).tobytes()
        if comp not in cache:
            lam, k, _ = ungapped_karlin_for_query(q, matrix)
            cache[comp] = (normalized_cutoff_to_nominal(ungapped_bits, lam),
                           normalized_to_nominal(trigger_bits, lam, k))
        cut[i], trig[i] = cache[comp]
    return cut, trig
