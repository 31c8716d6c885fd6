"""Writes the golden hit tables under tests/golden/reference_hits/: for every
case of tests/reference_hits.py, the tabular output of the reference's own
search on that case's inputs.

Each case's database is built by the reference's `ghostz db` (-C T or F,
-L 10, -s 39, -l chunk bytes where the case sets it) and searched by the
reference's GPU aligner, `ghostz-gpu aln -g 1 -a 4` (the reference's host
code compiled unchanged, its device operators computed on the CPU by the
reference's CPU arithmetic: oracle/ref_aln.py), with the `aln` defaults
(-v 1 -b 10 -F T, BLOSUM62, gap open 11, extension 1).  The script checks
that one and eight reference threads give the same table.  For the
reference's example files it also checks that the table is the one printed
in the reference's README and that the CPU aligner (`-g 0`) prints it too.

A case records the SHA-256 of the FASTA files it was made from (inputs
rebuilt by the seeded generators must match it), the sequence count of
every database chunk the reference made, and the command.  Run from the
repository root with the reference checkout present:

    GZ_REFERENCE_ROOT=<reference checkout> python tests/golden/make_reference_hit_tables.py
"""
import gzip
import json
import os
import struct
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for sub in ("ghostz-gpu_b200", "oracle", "tests"):
    sys.path.insert(0, os.path.join(ROOT, sub))

import ref_aln as R  # noqa: E402
import reference_hits as H  # noqa: E402

README_TABLE_START = "Example)"


def readme_table(reference_root):
    """The example table of the reference's README (tab separated)."""
    with open(os.path.join(reference_root, "README.md"), encoding="latin-1") as f:
        text = f.read()
    block = text.split(README_TABLE_START, 1)[1].split("```")[1]
    return [line for line in block.splitlines() if line.strip()]


def chunk_counts(prefix):
    """Sequences per chunk from the reference's <db>.inf and <db>_<k>.inf
    (Database::SaveInformation / DatabaseChunk: the first uint32 of a
    chunk's .inf is its sequence count)."""
    with open(prefix + ".inf", "rb") as f:
        number_chunks = struct.unpack("<I", f.read(4))[0]
    counts = []
    for k in range(number_chunks):
        with open(f"{prefix}_{k}.inf", "rb") as f:
            counts.append(struct.unpack("<I", f.read(4))[0])
    return counts


def run_case(name, reference_root):
    spec = H.CASES[name]
    stored = None
    if spec["kind"] == "fasta":
        with open(os.path.join(reference_root, "data", "db.fasta"), encoding="latin-1") as f:
            db_text = f.read()
        with open(os.path.join(reference_root, "data", "queries.fasta"), encoding="latin-1") as f:
            q_text = f.read()
        stored = {"db_fasta": db_text, "queries_fasta": q_text}
    inputs = H.case_inputs(name, stored)
    with tempfile.TemporaryDirectory() as tmp:
        db_fa, q_fa = os.path.join(tmp, "db.fa"), os.path.join(tmp, "q.fa")
        if stored is not None:
            open(db_fa, "w", encoding="latin-1").write(stored["db_fasta"])
            open(q_fa, "w", encoding="latin-1").write(stored["queries_fasta"])
        else:
            db_text, q_text = inputs.fasta()
            open(db_fa, "wb").write(db_text)
            open(q_fa, "wb").write(q_text)
        prefix = os.path.join(tmp, "db")
        R.build_database(db_fa, prefix, clustering=inputs.clustering,
                         chunk_bytes=inputs.chunk_bytes, threads=4)
        counts = chunk_counts(prefix)
        tables = []
        for threads in (1, 8):
            out = os.path.join(tmp, f"out{threads}.txt")
            R.align(q_fa, prefix, out, query_type=inputs.query_type, threads=threads,
                    gpu_aligner=True)
            tables.append(R.read_table(out))
        assert tables[0] == tables[1], f"{name}: 1 and 8 reference threads differ"
        lines = tables[0]
        if spec["kind"] == "fasta":
            cpu = os.path.join(tmp, "cpu.txt")
            R.align(q_fa, prefix, cpu, query_type=inputs.query_type)
            readme = readme_table(reference_root)
            assert [l.split() for l in lines] == [l.split() for l in readme], \
                f"{name}: the GPU aligner's table is not the README's"
            assert R.read_table(cpu) == lines, f"{name}: -g 0 and -g 1 differ"
    meta = {
        "name": name,
        "query_type": inputs.query_type,
        "clustering": inputs.clustering,
        "chunk_bytes": inputs.chunk_bytes,
        "chunk_sequence_counts": counts,
        "inputs_sha256": inputs.sha256(),
        "command": (f"ghostz db -C {'T' if inputs.clustering else 'F'} -L 10 -s 39"
                    + (f" -l {inputs.chunk_bytes}" if inputs.chunk_bytes else "")
                    + f"; ghostz-gpu aln -q {inputs.query_type} -t p -v 1 -b 10 -F T -g 1"),
        "lines": len(lines),
    }
    if stored is not None:
        meta.update(stored)
    os.makedirs(H.GOLDEN, exist_ok=True)
    with open(os.path.join(H.GOLDEN, name + ".json"), "w") as f:
        json.dump(meta, f, indent=1)
        f.write("\n")
    with gzip.GzipFile(os.path.join(H.GOLDEN, name + ".tsv.gz"), "wb", mtime=0) as f:
        f.write(("\n".join(lines) + "\n").encode("latin-1"))
    print(f"{name}: {len(lines)} lines, chunks {counts}")


def main():
    reference_root = os.environ.get("GZ_REFERENCE_ROOT")
    assert reference_root and os.path.isdir(os.path.join(reference_root, "src")), \
        "set GZ_REFERENCE_ROOT to the reference checkout"
    if not (R.available() and R.available(gpu_aligner=True)):
        R.build(reference_root)
    names = sys.argv[1:] or list(H.CASES)
    for name in names:
        run_case(name, reference_root)


if __name__ == "__main__":
    main()
