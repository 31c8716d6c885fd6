"""Per-query Karlin-Altschul statistics and cutoffs on the GPU against the
oracle's restatement of Statistics::CalculateUngappedKarlinParameters, bit
for bit (float lambda, K, H and the integer cutoffs)."""
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


def _layout(seqs):
    offsets = np.zeros(len(seqs), np.uint64)
    lengths = np.array([len(s) for s in seqs], np.uint32)
    if len(seqs) > 1:
        offsets[1:] = np.cumsum(lengths)[:-1]
    codes = np.concatenate(seqs).astype(np.uint8) if seqs else np.zeros(0, np.uint8)
    return codes, offsets, lengths


def _cases(oracle, seed):
    rng = np.random.default_rng(seed)
    db = W.make_database(60, seed + 1)
    reads = W.make_reads(db, 300, seed + 2)
    cases = [np.concatenate([[25], W.random_residues(rng, int(rng.integers(1, 4000))), [25]])
             for _ in range(400)]
    cases += [oracle.translate_query(reads.read(r), 25) for r in range(reads.number)]
    for _ in range(300):
        letters = rng.choice(25, size=int(rng.integers(1, 6)), replace=False)
        body = rng.choice(letters, size=int(rng.integers(1, 400)))
        cases.append(np.concatenate([[25], body, [25]]))
    # low-complexity queries whose K series needs more rounds (poly-S: 31 and
    # 32 rounds) than the first pass holds, so the second pass finishes them
    for n in (1000, 5000):
        cases.append(np.concatenate([[25], np.full(n, 15), [25]]))
    cases.append(np.array([25, 25]))          # an empty query
    cases.append(np.full(50, 24))             # only unknown letters, no delimiters
    return [np.asarray(c, np.uint8) for c in cases]


@pytest.mark.parametrize("seed", [50, 51])
def test_karlin_cutoffs_match_oracle(native, oracle, params, seed):
    cases = _cases(oracle, seed)
    codes, offsets, lengths = _layout(cases)
    cut, trig, kar = native.query_karlin_cutoffs(codes, offsets, lengths)
    for i, q in enumerate(cases):
        lam, k, h, c, t = oracle.query_karlin(params, q)
        assert (np.float32(lam), np.float32(k), np.float32(h)) == tuple(kar[i]), i
        assert (int(cut[i]), int(trig[i])) == (c, t), i


def test_karlin_cutoffs_other_bits(native, oracle, params):
    cases = _cases(oracle, 52)[:200]
    codes, offsets, lengths = _layout(cases)
    cut, trig, _ = native.query_karlin_cutoffs(codes, offsets, lengths, ungapped_bits=10.0,
                                               trigger_bits=30.0)
    for i, q in enumerate(cases):
        _, _, _, c, t = oracle.query_karlin(params, q, 10.0, 30.0)
        assert (int(cut[i]), int(trig[i])) == (c, t), i


def test_translated_reads_prepared_on_gpu(native, oracle):
    """Translation then cutoffs, both on the device, give the queries the
    host path builds."""
    db = W.make_database(300, 55)
    reads = W.make_reads(db, 500, 56)
    codes, offs, lens = native.translate_reads(reads.dna, reads.offsets, P.DELIMITER)
    cut, trig, _ = native.query_karlin_cutoffs(codes, offs, lens)
    q = W.translated_queries(codes, offs, lens)
    assert np.array_equal(cut, q.cutoffs) and np.array_equal(trig, q.triggers)
