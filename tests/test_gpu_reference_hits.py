"""The library's GPU search against the reference's own search: for every
golden case (tests/golden/reference_hits/: the tabular output of the
reference's GPU aligner compiled from its sources, on config-1 sized
protein, translated-read, four-chunk and unclustered workloads and on the
reference's README example), the hit table written from the GPU path --
query preparation, presearch of every chunk, build results, final order --
equals the reference's line for line."""
import pytest

import reference_hits as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gzb import native
    native.lib()
    return torch


def _check(got, exp):
    assert len(got) == len(exp)
    for i, (g, e) in enumerate(zip(got, exp)):
        assert g == e, (i, g, e)


@pytest.mark.parametrize("name", list(H.CASES))
def test_gpu_hit_table_matches_reference(gpu, name):
    meta = H.load_meta(name)
    inputs = H.case_inputs(name)
    assert inputs.sha256() == meta["inputs_sha256"]
    got = H.engine_hit_table(inputs, meta["chunk_sequence_counts"])
    _check(got, H.load_table(name))


def test_gpu_hit_table_graph_mode_config1(gpu):
    """The headline mode (one CUDA graph per chunk) on the 20,000-protein x
    1,000-query case."""
    name = "protein-1k-x-20k"
    meta = H.load_meta(name)
    got = H.engine_hit_table(H.case_inputs(name), meta["chunk_sequence_counts"], graph=True)
    _check(got, H.load_table(name))


def test_gpu_hit_table_plain_schedule_four_chunks(gpu):
    """The plain (static, one launch per stage) schedule on the four-chunk
    case."""
    from gzb import native as N
    name = "protein-300-x-20k-4chunks"
    meta = H.load_meta(name)
    got = H.engine_hit_table(H.case_inputs(name), meta["chunk_sequence_counts"],
                             schedule=N.SCHEDULE_PLAIN)
    _check(got, H.load_table(name))
