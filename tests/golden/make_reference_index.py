"""Writes reference_index_80.sdp: the reference's own seed-searcher index
file (SeedSearcherDatabaseParameters::Save,
src/seed_searcher_database_parameters.cpp:363-376) of the seeded
80-sequence chunk `chunk()` under the default `aln` parameters, produced
by the reference's compiled units (oracle/_ref).  Run from the repository
root with the reference checkout present:

    python tests/golden/make_reference_index.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for sub in ("ghostz-gpu_b200", "oracle"):
    sys.path.insert(0, os.path.join(ROOT, sub))

FIXTURE = os.path.join(HERE, "reference_index_80.sdp")


def chunk():
    """40 random proteins (median length 80) followed by a 90 %-identity
    copy of each without indels, so that windows cluster."""
    import numpy as np
    from gzb import params as P
    from gzb import workload as W
    base = W.make_database(40, 63, median=80)
    rng = np.random.default_rng(64)
    seqs = [base.codes[base.offsets[i]:base.offsets[i + 1] - 1] for i in range(40)]
    seqs += [W.mutate(rng, s, 0.9, indel_p=0.0) for s in seqs]
    codes = [np.array([P.DELIMITER], np.uint8)]
    offsets = []
    at = 1
    for s in seqs:
        offsets.append(at)
        codes += [np.asarray(s, np.uint8), np.array([P.DELIMITER], np.uint8)]
        at += len(s) + 1
    offsets.append(at)
    return W.Database(codes=np.concatenate(codes), offsets=np.array(offsets, np.uint32),
                      number_sequences=len(seqs))


def main():
    import oracle as O
    from gzb import params as P
    if not os.path.exists(O.REF_LIB):
        O.build(ref=True)
    ref = O.Reference()
    h = ref.db_index(P.make_params(), chunk().codes)
    try:
        data = ref.save_index(h)
    finally:
        ref.free_index(h)
    with open(FIXTURE, "wb") as f:
        f.write(data.tobytes())
    print(f"{FIXTURE}: {len(data)} bytes")


if __name__ == "__main__":
    main()
