"""Runs the reference's own programs (test infrastructure only).

* ``oracle/_ref/ghostz`` is GHOSTZ-GPU's `ghostz` program compiled from the
  reference checkout without -DGPU (`make -C oracle aln REF_ROOT=...`): its
  `db` command builds a database (src/database_build_main.cpp) and its `aln`
  command runs the CPU Aligner (`-g 0`, src/aligner.cpp).
* ``oracle/_ref/ghostz-gpu-host`` is the same program built with -DGPU
  (`make -C oracle alngpu`): `aln -g 1` runs the reference's GPU aligner
  (src/aligner_gpu.cpp, src/aligner_gpu_presearch_thread.cpp,
  src/seed_searcher_gpu*.cpp, src/gpu_stream_*.cpp) unchanged, its three
  device operators computed on the CPU by the reference's CPU arithmetic
  (refgpu/host_operators.cpp).  Its tabular output
  (AlignerCommon::WriteOutput, src/aligner_common.h:344-394) is the hit table
  the GPU path must reproduce.

The `-g 0` aligner is not the GPU path's oracle line for line:
AlignerPresearchThread::Extend (src/aligner_presearch_thread.cpp:320-364)
adds to an uninitialised end coordinate, which reorders ties in AddResults,
and AlignerBuildResultsThread counts mismatches along a path whose reverse
half is reversed twice, so the hit a tie keeps shows in the mismatch column.

The tests use these programs to make and check golden hit tables, and the
benchmark's reference arm times `ghostz aln`; the engine never calls them.
"""
from __future__ import annotations

import os
import subprocess
import time

HERE = os.path.dirname(os.path.abspath(__file__))
GHOSTZ = os.path.join(HERE, "_ref", "ghostz")
GHOSTZ_GPU_HOST = os.path.join(HERE, "_ref", "ghostz-gpu-host")
PROTEIN_LETTERS = "ARNDCQEGHILKMFPSTWYVBJZ*X"


def available(gpu_aligner: bool = False) -> bool:
    return os.access(GHOSTZ_GPU_HOST if gpu_aligner else GHOSTZ, os.X_OK)


def build(reference_root: str) -> None:
    """Compile _ref/ghostz and _ref/ghostz-gpu-host from a reference checkout."""
    subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "aln", "alngpu",
                           f"REF_ROOT={reference_root}"])


def letters(codes) -> bytes:
    """Residue codes (0-24) as protein letters."""
    table = PROTEIN_LETTERS.encode()
    return bytes(table[int(c)] for c in codes)


def write_fasta(path, names, sequences, width=60):
    """FASTA file of `sequences` (bytes of letters or bases) named `names`."""
    with open(path, "wb") as f:
        for name, seq in zip(names, sequences):
            f.write(b">" + name.encode() + b"\n")
            for i in range(0, max(len(seq), 1), width):
                f.write(bytes(seq[i:i + width]) + b"\n")


def build_database(fasta, prefix, clustering=True, chunk_bytes=None,
                   subsequence_length=10, seed_threshold=39, threads=1):
    """`ghostz db`: returns the seconds it took."""
    cmd = [GHOSTZ, "db", "-i", fasta, "-o", prefix, "-C", "T" if clustering else "F",
           "-L", str(subsequence_length), "-s", str(seed_threshold), "-a", str(threads)]
    if chunk_bytes is not None:
        cmd += ["-l", str(int(chunk_bytes))]
    t0 = time.perf_counter()
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return time.perf_counter() - t0


def align(queries_fasta, prefix, out_path, query_type="p", db_type="p",
          max_per_subject=1, max_per_query=10, filter=True, threads=1,
          gpu_aligner=False):
    """`ghostz aln`: the CPU Aligner (-g 0), or with gpu_aligner=True the
    reference's GPU aligner on its CPU stand-in operators (-g 1); returns the
    seconds it took."""
    cmd = [GHOSTZ_GPU_HOST if gpu_aligner else GHOSTZ, "aln", "-i", queries_fasta, "-d",
           prefix, "-o", out_path, "-q", query_type, "-t", db_type, "-v",
           str(max_per_subject), "-b", str(max_per_query), "-F", "T" if filter else "F",
           "-a", str(threads)]
    if gpu_aligner:
        cmd += ["-g", "1"]
    t0 = time.perf_counter()
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return time.perf_counter() - t0


def read_table(path):
    with open(path, "r", encoding="latin-1") as f:
        return f.read().splitlines()
