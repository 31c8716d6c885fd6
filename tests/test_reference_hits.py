"""The oracle's restatement of the whole search path against the reference's
own search: for every golden case (tests/golden/reference_hits/, made by the
reference's GPU aligner compiled from its sources), the hit table the CPU
oracle composes -- query preparation, each chunk's seed search, ungapped and
gapped extension, chain filter and top-b merge in chunk order, the build
results step, the final order -- equals the reference's line for line."""
import os

import pytest

import reference_hits as H


@pytest.mark.parametrize("name", list(H.CASES))
def test_case_inputs_are_the_ones_the_reference_searched(name):
    meta = H.load_meta(name)
    inputs = H.case_inputs(name)
    assert inputs.sha256() == meta["inputs_sha256"]
    assert sum(meta["chunk_sequence_counts"]) == len(inputs.subject_sequences)
    assert len(H.load_table(name)) == meta["lines"] > 0


@pytest.mark.parametrize("name", list(H.CASES))
def test_oracle_hit_table_matches_reference(oracle, name):
    meta = H.load_meta(name)
    inputs = H.case_inputs(name)
    got = H.oracle_hit_table(oracle, inputs, meta["chunk_sequence_counts"])
    exp = H.load_table(name)
    assert len(got) == len(exp)
    for i, (g, e) in enumerate(zip(got, exp)):
        assert g == e, (i, g, e)


def test_readme_case_is_the_readme_table():
    """The example case's table is the one the reference's README prints
    (query0 ... query4 against subject0 and subject6)."""
    lines = H.load_table("readme")
    assert [l.split("\t")[:2] for l in lines][:2] == [["query0", "subject0"],
                                                      ["query0", "subject6"]]
    assert lines[0].split("\t")[2:] == ["100", "25", "0", "0", "1", "75", "1", "25",
                                        "2.75456e-15", "60.4622"]


def test_reference_program_reproduces_readme_case(tmp_path):
    """Where the reference's programs are built (oracle/_ref), they still
    print the stored table for the example case."""
    import ref_aln as R
    if not R.available(gpu_aligner=True):
        pytest.skip("reference programs not built here")
    meta = H.load_meta("readme")
    db_fa, q_fa = tmp_path / "db.fa", tmp_path / "q.fa"
    db_fa.write_text(meta["db_fasta"], encoding="latin-1")
    q_fa.write_text(meta["queries_fasta"], encoding="latin-1")
    R.build_database(str(db_fa), str(tmp_path / "db"))
    R.align(str(q_fa), str(tmp_path / "db"), str(tmp_path / "out.txt"), query_type="d",
            gpu_aligner=True)
    assert R.read_table(str(tmp_path / "out.txt")) == H.load_table("readme")
