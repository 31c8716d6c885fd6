"""GHOSTZ-GPU's own program with this library as its device layer: the
reference's host sources compiled unchanged and linked with
ghostz-gpu_b200/adapters/reference_device_layer.cu in place of its CUDA files
(make -C ghostz-gpu_b200/adapters REF_ROOT=<reference checkout>).  Its
`db` builds each golden case's database and its `aln -g 1` -- AlignerGpu,
its presearch threads, SeedSearcherGpu and the stream controller and runner
driving this library's kernels -- must print the reference's own hit table
(tests/golden/reference_hits/) line for line."""
import os
import subprocess

import pytest

import reference_hits as H

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROGRAM = os.path.join(ROOT, "ghostz-gpu_b200", "adapters", "_build", "ghostz-gpu-b200")


@pytest.fixture(scope="module")
def program():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.access(PROGRAM, os.X_OK):
        pytest.skip("the reference program over this library is not built here")
    return PROGRAM


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (cmd, r.stdout[-2000:], r.stderr[-2000:])


@pytest.mark.parametrize("name", list(H.CASES))
def test_reference_aligner_on_this_library(program, tmp_path, name):
    meta = H.load_meta(name)
    inputs = H.case_inputs(name)
    assert inputs.sha256() == meta["inputs_sha256"]
    db_text, q_text = inputs.fasta()
    if "db_fasta" in meta:
        db_text = meta["db_fasta"].encode("latin-1")
        q_text = meta["queries_fasta"].encode("latin-1")
    (tmp_path / "db.fa").write_bytes(db_text)
    (tmp_path / "q.fa").write_bytes(q_text)
    prefix = str(tmp_path / "db")
    cmd = [program, "db", "-i", str(tmp_path / "db.fa"), "-o", prefix,
           "-C", "T" if inputs.clustering else "F", "-L", "10", "-s", "39", "-a", "4"]
    if inputs.chunk_bytes:
        cmd += ["-l", str(inputs.chunk_bytes)]
    _run(cmd)
    out = str(tmp_path / "out.txt")
    _run([program, "aln", "-i", str(tmp_path / "q.fa"), "-d", prefix, "-o", out,
          "-q", inputs.query_type, "-t", "p", "-v", "1", "-b", "10", "-F", "T", "-a", "4",
          "-g", "1"])
    with open(out, encoding="latin-1") as f:
        got = f.read().splitlines()
    exp = H.load_table(name)
    assert len(got) == len(exp)
    for i, (g, e) in enumerate(zip(got, exp)):
        assert g == e, (i, g, e)
