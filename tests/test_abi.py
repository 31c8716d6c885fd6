"""The C ABI library builds, loads without a GPU and exports every function
the public header declares; error reporting works without a device."""
import ctypes
import os

import pytest


def test_library_exports_header_symbols():
    from gzb import build as B
    from gzb import native as N
    if not os.path.exists(B.LIB):
        B.build()
    lib = ctypes.CDLL(B.LIB)
    declared = N.symbols_declared_in_header()
    assert len(declared) >= 35
    missing = [s for s in declared if not hasattr(lib, s)]
    assert missing == []


def test_error_strings_without_device():
    from gzb import native as N
    L = N.lib()
    assert L.gzb_error_string(0).decode() == "ok"
    assert "invalid" in L.gzb_error_string(1).decode()
    h = ctypes.c_void_p()
    assert L.gzb_distance_calculator_create(ctypes.byref(h)) == 0
    # using a handle before set-up reports GZB_ERR_INVALID with a message
    rc = L.gzb_distance_calculator_calculate_distances_async(
        h, 1, None, None, None, None, None, None, None)
    assert rc == 1 and b"not set up" in L.gzb_last_error()
    assert L.gzb_distance_calculator_destroy(h) == 0


def test_engine_create_reports_missing_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("device present")
    from gzb import native as N
    with pytest.raises(N.GzbError):
        N.PresearchEngine(0)


def test_params_record_matches_header_layout(tmp_path):
    import subprocess
    from gzb import params as P
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "size.c"
    src.write_text('#include "ghostz_b200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu\\n", sizeof(gzb_params), '
                   'offsetof(gzb_params, code_scores), sizeof(gzb_result));return 0;}\n')
    exe = tmp_path / "size"
    subprocess.check_call(["gcc", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)])
    size, off, rsize = map(int, subprocess.check_output([str(exe)]).split())
    assert size == P.PARAMS_DTYPE.itemsize
    assert off == P.PARAMS_DTYPE.fields["code_scores"][1]
    from gzb import native as N
    assert rsize == N.RESULT_DTYPE.itemsize


def test_cpp_adapters_compile_and_link(tmp_path):
    """The header-only C++ classes with the reference's names compile and
    link against the library (no GPU needed: nothing is called)."""
    import subprocess
    from gzb import build as B
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "use.cpp"
    src.write_text(
        '#include "ghostz_gpu_adapters.h"\n'
        'using namespace ghostz_b200;\n'
        'int run(cudaStream_t s) {\n'
        '  DistanceCalculatorGpu d; UngappedExtenderGpu u; GappedExtenderGpu g;\n'
        '  uint32_t *p = 0; char *f = 0; int *i = 0;\n'
        '  d.SetSubsequenceLength(10);\n'
        '  u.ExtendWithTriggerAsync(0, p, p, p, f, p, p, p, f, i, s);\n'
        '  return g.ExtendOneSideScoreOnlyAsync(0, true, p, p, i, p, p, i, s);\n'
        '}\n'
        'int load(gzb_engine *e, const gzb_params &prm, std::istream &in, cudaStream_t s) {\n'
        '  return LoadChunkWithReferenceIndex(e, prm, 0, 0, 0, 0, 0, in, s);\n'
        '}\n'
        'int main() { return 0; }\n')
    exe = tmp_path / "use"
    subprocess.check_call([
        "g++", "-std=c++11", "-I", os.path.join(root, "include"),
        "-I", os.path.join(root, "ghostz-gpu_b200", "adapters"),
        "-I", "/usr/local/cuda/include", str(src), "-o", str(exe),
        B.LIB, "-Wl,-rpath," + os.path.dirname(B.LIB)])


def test_tile_parameters_validate_without_device():
    from gzb import native as N
    L = N.lib()
    v = ctypes.c_int()
    for which in (N.TILE_BOOK_THRESHOLD, N.TILE_GAPPED_KERNEL, N.TILE_ORDER,
                  N.TILE_SEED_WALKER, N.TILE_BAND_WIDTH):
        assert L.gzb_get_tile_parameter(which, ctypes.byref(v)) == 0
        keep = v.value
        assert L.gzb_set_tile_parameter(which, keep) == 0
    assert L.gzb_set_tile_parameter(N.TILE_BOOK_THRESHOLD, 0) == 1
    assert L.gzb_set_tile_parameter(N.TILE_BOOK_THRESHOLD, 33) == 1
    assert L.gzb_set_tile_parameter(N.TILE_GAPPED_KERNEL, 9) == 1
    assert b"none of" in L.gzb_last_error()
    assert L.gzb_set_tile_parameter(N.TILE_ORDER, 2) == 1
    assert L.gzb_set_tile_parameter(N.TILE_SEED_WALKER, 2) == 1
    assert L.gzb_get_tile_parameter(N.TILE_BAND_WIDTH, ctypes.byref(v)) == 0 and v.value == 64
    for bad in (0, 16, 48, 96, 256):
        assert L.gzb_set_tile_parameter(N.TILE_BAND_WIDTH, bad) == 1
    assert L.gzb_set_tile_parameter(7, 1) == 1
    assert L.gzb_get_tile_parameter(7, ctypes.byref(v)) == 1


def test_translated_layout_without_device(oracle):
    import numpy as np
    from gzb import native as N
    for n in list(range(0, 50)) + [150, 151, 152, 99999]:
        assert N.translated_query_length(n) == oracle.L.gzo_translated_length(n)
    lengths = np.array([150, 2, 0, 7, 3], np.uint32)
    offs, ql, total = N.translated_layout(lengths)
    assert list(ql) == [7 + 6 * 50, 2, 2, 7 + 12, 13]
    # consecutive queries share a delimiter
    assert list(offs) == [0, 306, 307, 308, 326] and total == 326 + 13
    # the device entry point refuses null buffers before touching a device
    rc = N.lib().gzb_translate_dna_queries(None, None, None, 1, None, 25, None, None)
    assert rc == 1


def test_karlin_cutoffs_validate_without_device():
    import numpy as np
    from gzb import native as N
    from gzb import params as P
    m = P.blosum62()
    L = N.lib()
    f = L.gzb_query_karlin_cutoffs
    # zero queries: validated and returns before touching a device
    assert f(None, None, None, 0, N.hptr(np.ascontiguousarray(m, np.int32)), 25, 7.0, 22.0,
             None, None, None, None) == 0
    assert f(None, None, None, 0, None, 25, 7.0, 22.0, None, None, None, None) == 1
    wide = np.ascontiguousarray(m * 3, np.int32)  # score range 45 > 31
    assert f(None, None, None, 0, N.hptr(wide), 25, 7.0, 22.0, None, None, None, None) == 4
    assert f(None, None, None, 1, N.hptr(np.ascontiguousarray(m, np.int32)), 25, 7.0, 22.0,
             None, None, None, None) == 1


def test_hit_statistics_without_device(oracle):
    """The library's hit-table statistics (host code) equal the oracle's."""
    import numpy as np
    from gzb import native as N
    karlin = N.gapped_karlin_parameters()
    assert np.float32(karlin[0]) == np.float32(0.267) and np.float32(karlin[1]) == np.float32(0.041)
    rng = np.random.default_rng(82)
    for _ in range(300):
        ql, dl = int(rng.integers(1, 10000)), int(rng.integers(10, 10**10))
        ns = int(rng.integers(1, min(dl, 10**7)))
        score = int(rng.integers(0, 3000))
        space = N.search_space(ql, dl, ns, karlin)
        exp = oracle.hit_statistics(ql, dl, ns, score)
        assert space == exp[0]
        assert N.evalue(score, space, karlin) == exp[1]
        assert np.float32(N.bit_score(score, karlin)) == np.float32(exp[2])
    for n in (3, 75, 150, 1000):
        slot = n // 3 + 1
        for pos in range(1, 6 * slot):
            if pos % slot == 0:
                continue
            assert (N.lib().gzb_translated_real_start(pos, n),
                    N.lib().gzb_translated_real_end(pos, n)) == oracle.translated_real(pos, n)
    import pytest
    with pytest.raises(N.GzbError):
        N.gapped_karlin_parameters("BLOSUM62", 10, 1)
