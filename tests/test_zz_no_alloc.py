"""The allocation-free gapped extension entry point.

It exists for callers that cannot call cudaMalloc (a host runtime that owns
every device buffer, or a latency-critical loop that cannot take an
allocation's device synchronisation).  These tests call it through the C
ABI and require exactly the results of the regular entry point, which
allocates its own scratch, on two calls in a row -- the shared scratch array
keeps the previous call's contents, so the second call checks that nothing
stale leaks into it -- and a sample of them against the CPU oracle.  A call
whose extension outgrows the fixed fallback band must report
GZB_ERR_OVERFLOW, and the next call must again match the regular entry
point.  The file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_EXTENSIONS = 1 << 20


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gzb import native
    native.lib()
    return torch


def _workload(seed, n, lo, hi):
    from gzb import workload as W
    rng = np.random.default_rng(seed)
    A, B = [], []
    for _ in range(n):
        a = W.random_residues(rng, int(rng.integers(lo, hi)))
        A.append(a)
        B.append(W.mutate(rng, a, rng.uniform(0.3, 1.0)))

    def concat(seqs):
        out, starts, pos = [np.array([25], np.uint8)], [], 1
        for s in seqs:
            starts.append(pos)
            out += [s, np.array([25], np.uint8)]
            pos += len(s) + 1
        return np.concatenate(out), starts

    qc, qs = concat(A)
    dc, ds = concat(B)
    qpos = np.array([qs[i] + int(rng.integers(0, len(A[i]))) for i in range(n)], np.uint32)
    dpos = np.array([ds[i] + min(int(qpos[i] - qs[i]), len(B[i]) - 1) for i in range(n)],
                    np.uint32)
    return qc, dc, qpos, dpos


def _regular(torch, qa, da, tm, qpos, dpos, reverse, cutoff):
    from gzb import native as N
    g = N.GappedExtenderGpu()
    g.SetQueries(25, qa)
    g.SetDatabase(da)
    g.SetScoreParameters(tm, 25, 11, 1, cutoff)
    n = len(qpos)
    hq, hd, hs = qpos.copy(), dpos.copy(), np.zeros(n, np.int32)
    dq = torch.from_numpy(qpos.view(np.int32).copy()).cuda()
    dd = torch.from_numpy(dpos.view(np.int32).copy()).cuda()
    ds = torch.zeros(n, dtype=torch.int32, device="cuda")
    g.ExtendOneSideScoreOnlyAsync(n, reverse, hq, hd, hs, dq, dd, ds)
    torch.cuda.synchronize()
    g.close()
    return hs, hq, hd


def _noalloc(torch, qa, da, tm, qpos, dpos, reverse, cutoff):
    from gzb import native as N
    n = len(qpos)
    dq = torch.from_numpy(qpos.view(np.int32).copy()).cuda()
    dd = torch.from_numpy(dpos.view(np.int32).copy()).cuda()
    ds = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = N.lib().gzb_gapped_extend_one_side_score_only_noalloc(
        C.c_void_p(qa), C.c_void_p(da), C.c_uint8(25), C.c_void_p(tm.data_ptr()),
        C.c_uint32(25), 11, 1, int(cutoff), C.c_size_t(n), int(reverse),
        C.c_void_p(dq.data_ptr()), C.c_void_p(dd.data_ptr()), C.c_void_p(ds.data_ptr()),
        C.c_void_p(stream.cuda_stream))
    N.check(rc)
    torch.cuda.synchronize()
    return (ds.cpu().numpy(), dq.cpu().numpy().view(np.uint32),
            dd.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("cutoff,lo,hi", [(26, 30, 900), (2000, 20, 300), (2**31 - 1, 20, 400)])
def test_noalloc_matches_regular_entry_point(torch_cuda, oracle, cutoff, lo, hi):
    from gzb import native as N
    from gzb import params as P
    torch = torch_cuda
    p = P.make_params()
    N.lib().gzb_gapped_extend_one_side_score_only_noalloc.restype = C.c_int
    qc, dc, qpos, dpos = _workload(31 + cutoff % 7, 600, lo, hi)
    tq, qa = N.device_sequence(qc, 25)
    td, da = N.device_sequence(dc, 25)
    tm = N.device_matrix(P.blosum62())
    for reverse in (False, True):
        exp = _regular(torch, qa, da, tm, qpos, dpos, reverse, cutoff)
        for _ in range(2):  # two calls in a row share the scratch array
            got = _noalloc(torch, qa, da, tm, qpos, dpos, reverse, cutoff)
            for g, e in zip(got, exp):
                assert np.array_equal(g, e)
        # and a sample against the oracle's GappedExtender restatement
        for i in range(0, len(qpos), 37):
            es, eq, ed, _ = oracle.gapped_one_side(p, qc, int(qpos[i]), dc, int(dpos[i]),
                                                   reverse, cutoff)
            assert (int(got[0][i]), int(got[1][i]), int(got[2][i])) == \
                (es, int(qpos[i]) + eq, int(dpos[i]) + ed), (i, reverse)


def test_noalloc_reports_too_wide_bands_then_recovers(torch_cuda):
    """One near-identical 9,000-residue pair with an X-drop that prunes
    nothing needs a band wider than the 8,192-column fallback: the call
    returns GZB_ERR_OVERFLOW (its position and score buffers are then
    undefined), and the next call, on other extensions, matches the regular
    entry point."""
    from gzb import native as N
    from gzb import params as P
    from gzb import workload as W
    torch = torch_cuda
    L = N.lib()
    L.gzb_gapped_extend_one_side_score_only_noalloc.restype = C.c_int
    rng = np.random.default_rng(909)
    a = W.random_residues(rng, 9000)
    b = W.mutate(rng, a, 0.95, indel_p=0.0)
    qc = np.concatenate([[25], a, [25]]).astype(np.uint8)
    dc = np.concatenate([[25], b, [25]]).astype(np.uint8)
    tq, qa = N.device_sequence(qc, 25)
    td, da = N.device_sequence(dc, 25)
    tm = N.device_matrix(P.blosum62())
    dq = torch.tensor([1], dtype=torch.int32, device="cuda")
    dd = torch.tensor([1], dtype=torch.int32, device="cuda")
    ds = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = L.gzb_gapped_extend_one_side_score_only_noalloc(
        C.c_void_p(qa), C.c_void_p(da), C.c_uint8(25), C.c_void_p(tm.data_ptr()),
        C.c_uint32(25), 11, 1, 2**31 - 1, C.c_size_t(1), 0, C.c_void_p(dq.data_ptr()),
        C.c_void_p(dd.data_ptr()), C.c_void_p(ds.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == 4  # GZB_ERR_OVERFLOW
    assert b"band wider" in L.gzb_last_error()
    qc2, dc2, qpos, dpos = _workload(57, 300, 30, 600)
    tq2, qa2 = N.device_sequence(qc2, 25)
    td2, da2 = N.device_sequence(dc2, 25)
    for reverse in (False, True):
        exp = _regular(torch, qa2, da2, tm, qpos, dpos, reverse, 26)
        got = _noalloc(torch, qa2, da2, tm, qpos, dpos, reverse, 26)
        for g, e in zip(got, exp):
            assert np.array_equal(g, e)


def test_noalloc_rejects_oversized_calls(torch_cuda):
    from gzb import native as N
    L = N.lib()
    rc = L.gzb_gapped_extend_one_side_score_only_noalloc(
        C.c_void_p(1), C.c_void_p(1), C.c_uint8(25), C.c_void_p(1), C.c_uint32(25), 11, 1, 26,
        C.c_size_t(MAX_EXTENSIONS + 1), 0, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None)
    assert rc == 4  # GZB_ERR_OVERFLOW, before any device work
    assert b"exceed" in L.gzb_last_error()
