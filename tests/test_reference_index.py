"""The reference's on-disk seed-searcher index of a chunk (the bytes of its
.sdp file, written by the reference's own units here) converted to this
library's index blob on the host: the blob's arrays equal the oracle's
index (itself pinned to the reference's), the representatives' windows are
the chunk's similarity windows, and files built with other parameters,
truncated or inconsistent are refused."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

NAMES = ("nc_keys", "nc_offsets", "nc_values", "rep_keys", "rep_offsets", "rep_positions",
         "rep_cluster_ids", "rep_windows", "member_offsets", "member_positions")
HEADER = 10 * 8
MAGIC = 0x3130584449425a47


def parse_blob(blob):
    h = [int(x) for x in blob[:HEADER].view(np.uint64)]
    magic, _, db_len, nseq, _, n_nc_keys, n_nc_values, n_rep_keys, n_reps, n_members = h
    sizes = (n_nc_keys, n_nc_keys + 1, n_nc_values, n_rep_keys, n_rep_keys + 1, n_reps, n_reps,
             n_reps, n_reps + 1, n_members)
    out = {"magic": magic, "db_len": db_len, "nseq": nseq}
    at = HEADER
    for i, (name, n) in enumerate(zip(NAMES, sizes)):
        width = 8 if name == "rep_windows" else 4
        out[name] = blob[at:at + n * width].view(np.uint64 if width == 8 else np.uint32).copy()
        at += (n * width + 7) // 8 * 8
    assert at == len(blob)
    return out


def windows(params, codes, positions):
    """Similarity codes of the L-window centred on each position, 4 bits per
    code, codes outside the chunk read as the delimiter."""
    L = int(params["subsequence_length"])
    half = L // 2
    sim = np.asarray(params["similarity_code_map"], np.uint64) & np.uint64(15)
    padded = np.concatenate([np.full(L, P.DELIMITER, np.uint8), codes,
                             np.full(L, P.DELIMITER, np.uint8)])
    out = np.zeros(len(positions), np.uint64)
    for t in range(L):
        c = padded[positions.astype(np.int64) - half + t + L]
        out |= sim[c] << np.uint64(4 * t)
    return out


@pytest.fixture(scope="module")
def native():
    from gzb import native as N
    return N


@pytest.mark.parametrize("clustering", [True, False])
def test_reference_index_file_becomes_the_device_blob(native, oracle, reference, clustering):
    params = P.make_params(clustering=clustering)
    db = W.make_database(400, 61, median=150)
    h = reference.db_index(params, db.codes)
    try:
        sdp = reference.save_index(h)
    finally:
        reference.free_index(h)
    blob = native.index_blob_from_reference(params, sdp, db)
    got = parse_blob(blob)
    assert got["magic"] == MAGIC and got["db_len"] == len(db.codes)
    assert got["nseq"] == db.number_sequences
    exp = oracle.db_index(params, db.codes)
    for name in ("nc_keys", "nc_offsets", "nc_values"):
        assert np.array_equal(got[name], exp[name]), name
    if clustering:
        for name in ("rep_keys", "rep_offsets", "rep_positions", "member_offsets",
                     "member_positions"):
            assert np.array_equal(got[name], exp[name]), name
        n = len(got["rep_positions"])
        assert n > 0 and len(got["member_positions"]) > 0
        assert np.array_equal(got["rep_cluster_ids"], np.arange(n, dtype=np.uint32))
        assert np.array_equal(got["rep_windows"],
                              windows(params, db.codes, got["rep_positions"]))
    else:
        assert len(got["rep_keys"]) == 0 and len(got["member_positions"]) == 0
        assert list(got["rep_offsets"]) == [0] and list(got["member_offsets"]) == [0]


def test_reference_index_file_refused_when_it_does_not_fit(native, reference):
    params = P.make_params()
    db = W.make_database(200, 62, median=120)
    h = reference.db_index(params, db.codes)
    try:
        sdp = reference.save_index(h)
    finally:
        reference.free_index(h)
    assert len(native.index_blob_from_reference(params, sdp, db)) > HEADER
    cases = {
        "truncated": (params, sdp[:-3]),
        "trailing bytes": (params, np.concatenate([sdp, [0]]).astype(np.uint8)),
        "other window": (P.make_params(subsequence_length=12), sdp),
        "other seed threshold": (P.make_params(seed_threshold=35), sdp),
        "without clustering": (P.make_params(clustering=False), sdp),
        "empty": (params, np.zeros(0, np.uint8)),
    }
    for what, (p, data) in cases.items():
        with pytest.raises(native.GzbError):
            native.index_blob_from_reference(p, data, db)
    # positions beyond the chunk: the same file against a shorter chunk
    short = W.Database(codes=db.codes[:len(db.codes) // 2].copy(),
                       offsets=db.offsets.copy(), number_sequences=db.number_sequences)
    with pytest.raises(native.GzbError, match="outside the chunk"):
        native.index_blob_from_reference(params, sdp, short)


def _golden():
    import importlib.util
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                        "make_reference_index.py")
    spec = importlib.util.spec_from_file_location("make_reference_index", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_golden_file_is_the_reference_index(reference):
    """The committed .sdp fixture is what the reference's units write for
    the fixture's chunk."""
    g = _golden()
    h = reference.db_index(P.make_params(), g.chunk().codes)
    try:
        data = reference.save_index(h).tobytes()
    finally:
        reference.free_index(h)
    with open(g.FIXTURE, "rb") as f:
        assert f.read() == data


def test_golden_file_converts_to_the_oracle_index(native, oracle):
    """The fixture (clustered: every protein has a 90 %-identity copy) gives
    the oracle's index arrays without the reference's units."""
    g = _golden()
    params = P.make_params()
    db = g.chunk()
    with open(g.FIXTURE, "rb") as f:
        got = parse_blob(native.index_blob_from_reference(params, f.read(), db))
    exp = oracle.db_index(params, db.codes)
    for name in ("nc_keys", "nc_offsets", "nc_values", "rep_keys", "rep_offsets",
                 "rep_positions", "member_offsets", "member_positions"):
        assert np.array_equal(got[name], exp[name]), name
    assert len(got["rep_positions"]) > 1000 and len(got["member_positions"]) > 1000
    assert np.array_equal(got["rep_windows"], windows(params, db.codes, got["rep_positions"]))


def test_common_parameter_file_gives_the_seed_parameters(native, reference):
    """The reference's .scp file of a database yields the seed-index fields
    of the parameters it was built with; the caller's other fields stay."""
    for kw in ({}, {"subsequence_length": 12, "seed_threshold": 35}):
        params = P.make_params(**kw)
        db = W.make_database(40, 65, median=80)
        h = reference.db_index(params, db.codes)
        try:
            scp = reference.save_common(h)
        finally:
            reference.free_index(h)
        blank = P.make_params()
        for f in ("delimiter", "subsequence_length", "map_size", "max_indexing_code",
                  "seed_threshold", "max_hash_length"):
            blank[f] = 0
        for f in ("similarity_code_map", "hash_code_map", "code_scores"):
            blank[f] = 0
        blank["gap_open"] = 7
        got = native.params_from_reference_common(scp, blank)
        for f in ("delimiter", "subsequence_length", "map_size", "max_indexing_code",
                  "seed_threshold", "max_hash_length", "similarity_code_map", "hash_code_map",
                  "code_scores"):
            assert np.array_equal(got[f], params[f]), f
        assert got["gap_open"] == 7
        with pytest.raises(native.GzbError):
            native.params_from_reference_common(scp[:-1], blank)


def test_c_caller_converts_the_golden_file(tmp_path):
    """A plain C program (the reference host's side of the boundary) reads
    the committed .sdp file, converts it through the C ABI and finds the
    blob's counts: the host entry points need nothing but the header and
    the library."""
    import os
    import subprocess
    from gzb import build as B
    g = _golden()
    params = P.make_params()
    db = g.chunk()
    codes, offsets = tmp_path / "codes.bin", tmp_path / "offsets.bin"
    prm = tmp_path / "params.bin"
    db.codes.astype(np.uint8).tofile(codes)
    db.offsets.astype(np.uint32).tofile(offsets)
    np.array([params]).tofile(prm)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "convert.c"
    src.write_text(r'''
#include <stdio.h>
#include <stdlib.h>
#include "ghostz_b200.h"
static void *slurp(const char *path, long *n) {
  FILE *f = fopen(path, "rb"); void *p; fseek(f, 0, SEEK_END); *n = ftell(f);
  fseek(f, 0, SEEK_SET); p = malloc(*n ? *n : 1); fread(p, 1, *n, f); fclose(f); return p;
}
int main(int argc, char **argv) {
  long ns, nc, no, np_;
  void *sdp = slurp(argv[1], &ns);
  unsigned char *codes = slurp(argv[2], &nc);
  unsigned int *offsets = slurp(argv[3], &no);
  gzb_params *p = slurp(argv[4], &np_);
  uint64_t n = 0;
  unsigned int nseq = (unsigned int)(no / 4 - 1);
  if (np_ != (long)sizeof(gzb_params)) return 3;
  if (gzb_index_blob_from_reference(p, sdp, ns, codes, nc, offsets, nseq, 0, 0, &n)) return 1;
  uint64_t *blob = malloc(n);
  if (gzb_index_blob_from_reference(p, sdp, ns, codes, nc, offsets, nseq, blob, n, &n)) return 2;
  /* header: magic, fingerprint, length, sequences, check, then the counts */
  printf("%llu %llu %llu %llu %llu\n", (unsigned long long)n, (unsigned long long)blob[2],
         (unsigned long long)blob[3], (unsigned long long)blob[8], (unsigned long long)blob[9]);
  return 0;
}
''')
    exe = tmp_path / "convert"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(root, "include"), str(src),
                           "-o", str(exe), B.LIB, "-Wl,-rpath," + os.path.dirname(B.LIB)])
    out = subprocess.run([str(exe), g.FIXTURE, str(codes), str(offsets), str(prm)],
                         capture_output=True, text=True, check=True).stdout.split()
    from gzb import native as N
    with open(g.FIXTURE, "rb") as f:
        blob = N.index_blob_from_reference(params, f.read(), db)
    got = parse_blob(blob)
    assert [int(x) for x in out] == [len(blob), len(db.codes), db.number_sequences,
                                     len(got["rep_positions"]), len(got["member_positions"])]
