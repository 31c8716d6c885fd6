"""Per-operator parity on the GPU: DistanceCalculatorGpu, UngappedExtenderGpu
and GappedExtenderGpu through the C ABI against the CPU oracle, bit for bit,
plus the reference GPU unit tests' known answers."""
import numpy as np
import pytest

from gzb import params as P
from gzb import workload as W

pytestmark = pytest.mark.gpu

INT_MAX = 2**31 - 1


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gzb import native
    native.lib()
    return torch


def _concat(seqs, delim):
    out = [np.array([delim], np.uint8)]
    starts = []
    pos = 1
    for s in seqs:
        starts.append(pos)
        out.append(np.asarray(s, np.uint8))
        out.append(np.array([delim], np.uint8))
        pos += len(s) + 1
    return np.concatenate(out), np.array(starts)


def _pairs(rng, n, lo=5, hi=600):
    A, B = [], []
    for _ in range(n):
        a = W.random_residues(rng, int(rng.integers(lo, hi)))
        b = W.mutate(rng, a, rng.uniform(0.25, 1.0))
        A.append(a)
        B.append(b)
    return A, B


def _gapped_gpu(torch, params, qcodes, dcodes, qpos, dpos, reverse, cutoff,
                matrix=None, nletters=None, delim=None):
    from gzb import native as N
    delim = int(params["delimiter"]) if delim is None else delim
    if matrix is None:
        nl = int(params["number_letters"])
        matrix = np.asarray(params["score_matrix"][: nl * nl]).reshape(nl, nl)
    nl = matrix.shape[0] if nletters is None else nletters
    tq, q_addr = N.device_sequence(qcodes, delim)
    td, d_addr = N.device_sequence(dcodes, delim)
    tm = N.device_matrix(matrix)
    g = N.GappedExtenderGpu()
    g.SetQueries(delim, q_addr)
    g.SetDatabase(d_addr)
    g.SetScoreParameters(tm, nl, int(params["gap_open"]), int(params["gap_extension"]), cutoff)
    n = len(qpos)
    hq = np.asarray(qpos, np.uint32).copy()
    hd = np.asarray(dpos, np.uint32).copy()
    hs = np.zeros(n, np.int32)
    dq = torch.from_numpy(hq.copy()).cuda()
    dd = torch.from_numpy(hd.copy()).cuda()
    ds = torch.zeros(n, dtype=torch.int32, device="cuda")
    g.ExtendOneSideScoreOnlyAsync(n, reverse, hq, hd, hs, dq, dd, ds)
    torch.cuda.synchronize()
    cells = g.Cells()
    g.close()
    return hs, hq, hd, cells


def _dna_params():
    m = np.full((4, 4), -1, np.int32)
    np.fill_diagonal(m, 2)
    p = P.make_params(matrix=m, gap_open=0, gap_extension=1)
    p["delimiter"] = 5
    return p, m


def _dna(s):
    return np.array([5] + ["ACGT".index(c) for c in s] + [5], np.uint8)


def test_gapped_known_answers(torch_cuda):
    # test/gapped_extender_gpu_test.cu:40-253
    p, m = _dna_params()
    s, q, d, _ = _gapped_gpu(torch_cuda, p, _dna("AGCAC"), _dna("AGCAG"), [1], [1], False, 0,
                             matrix=m, delim=5)
    assert (s[0], q[0], d[0]) == (8, 4, 4)
    a, b = _dna("AGTCAC"), _dna("AGCAG")
    s, q, d, _ = _gapped_gpu(torch_cuda, p, a, b, [1], [1], False, INT_MAX, matrix=m, delim=5)
    assert (s[0], q[0], d[0]) == (7, 5, 4)
    s, q, d, _ = _gapped_gpu(torch_cuda, p, a, b, [len(a) - 3], [len(b) - 3], True, INT_MAX,
                             matrix=m, delim=5)
    assert (s[0], q[0], d[0]) == (7, 1, 1)


@pytest.mark.parametrize("cutoff", [0, 5, 26, 60, 2000, INT_MAX])
@pytest.mark.parametrize("reverse", [False, True])
def test_gapped_matches_oracle(torch_cuda, oracle, params, cutoff, reverse):
    rng = np.random.default_rng(1000 + cutoff % 97 + (7 if reverse else 0))
    n = 400 if cutoff not in (2000, INT_MAX) else 120
    A, B = _pairs(rng, n, hi=600 if cutoff < 1000 else 250)
    qc, qs = _concat(A, 25)
    dc, ds = _concat(B, 25)
    qpos, dpos = [], []
    for i in range(n):
        pa = int(rng.integers(0, len(A[i])))
        pb = int(np.clip(pa + rng.integers(-4, 5), 0, len(B[i]) - 1))
        qpos.append(qs[i] + pa)
        dpos.append(ds[i] + pb)
    s, q, d, cells = _gapped_gpu(torch_cuda, params, qc, dc, qpos, dpos, reverse, cutoff)
    total = 0
    for i in range(n):
        es, eq, ed, ec = oracle.gapped_one_side(params, qc, qpos[i], dc, dpos[i], reverse, cutoff)
        total += ec
        assert (int(s[i]), int(q[i]), int(d[i])) == (es, int(qpos[i]) + eq, int(dpos[i]) + ed), (i, cutoff, reverse)
    assert cells == total


def test_gapped_long_homologs(torch_cuda, oracle, params):
    # long near-identical pairs at the presearch X-drop: wide, long bands
    rng = np.random.default_rng(77)
    A, B = _pairs(rng, 40, lo=2000, hi=8000)
    qc, qs = _concat(A, 25)
    dc, ds = _concat(B, 25)
    qpos = [qs[i] + len(A[i]) // 2 for i in range(40)]
    dpos = [ds[i] + len(A[i]) // 2 for i in range(40)]
    for rev in (False, True):
        s, q, d, cells = _gapped_gpu(torch_cuda, params, qc, dc, qpos, dpos, rev,
                                     int(params["gapped_cutoff"]))
        for i in range(40):
            es, eq, ed, _ = oracle.gapped_one_side(params, qc, qpos[i], dc, dpos[i], rev,
                                                   int(params["gapped_cutoff"]))
            assert (int(s[i]), int(q[i]), int(d[i])) == (es, int(qpos[i]) + eq, int(dpos[i]) + ed)


def test_ungapped_flags_match_oracle(torch_cuda, oracle, params):
    from gzb import native as N
    torch = torch_cuda
    rng = np.random.default_rng(5)
    A, B = _pairs(rng, 300, lo=10, hi=300)
    qc, qs = _concat(A, 25)
    dc, ds = _concat(B, 25)
    nq = len(A)
    cut = rng.integers(5, 25, nq).astype(np.int32)
    trig = rng.integers(10, 60, nq).astype(np.int32)
    seeds = []
    for i in range(nq):
        for _ in range(20):
            pa = int(rng.integers(0, len(A[i])))
            pb = int(np.clip(pa + rng.integers(-2, 3), 0, len(B[i]) - 1))
            seeds.append((i, qs[i] + pa, ds[i] + pb))
    qid = np.array([x[0] for x in seeds], np.uint32)
    qp = np.array([x[1] for x in seeds], np.uint32)
    dp = np.array([x[2] for x in seeds], np.uint32)
    tq, qa = N.device_sequence(qc, 25)
    td, da = N.device_sequence(dc, 25)
    tm = N.device_matrix(P.blosum62())
    tcut = torch.from_numpy(cut).cuda()
    ttrig = torch.from_numpy(trig).cuda()
    u = N.UngappedExtenderGpu()
    u.SetQueries(25, qa, tcut, ttrig)
    u.SetDatabase(da)
    u.SetScoreMatrix(tm, 25)
    n = len(seeds)
    flags = np.zeros(n, np.int8)
    d_qid = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_qp = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_fl = torch.zeros(n, dtype=torch.int8, device="cuda")
    u.ExtendWithTriggerAsync(n, qid, qp, dp, flags, d_qid, d_qp, d_dp, d_fl)
    torch.cuda.synchronize()
    exp = np.array([oracle.ungapped_with_trigger(params, qc, int(q), dc, int(d), cut[i],
                                                 trig[i]) > trig[i]
                    for (i, q, d) in seeds], np.int8)
    assert np.array_equal(flags, exp)
    assert 0 < exp.sum() < n


@pytest.mark.parametrize("L", [10, 7, 13, 16])
def test_distances_match_oracle(torch_cuda, oracle, L):
    """Windows up to 13 letters are read as aligned words, longer ones byte
    by byte: both give the reference's distances."""
    from gzb import native as N
    from gzb import params as P
    torch = torch_cuda
    params = P.make_params(subsequence_length=L)
    rng = np.random.default_rng(6 + L)
    a = W.random_residues(rng, 20000)
    b = a.copy()
    m = rng.random(len(b)) < 0.15
    b[m] = W.random_residues(rng, int(m.sum()))
    n = 50000
    c0 = rng.integers(L, len(a) - L, n).astype(np.uint32)
    c1 = np.clip(c0.astype(np.int64) + rng.integers(-2, 3, n), L, len(b) - L).astype(np.uint32)
    tq, qa = N.device_sequence(a, 25)
    td, da = N.device_sequence(b, 25)
    tmap = torch.from_numpy(np.asarray(params["similarity_code_map"]).copy()).cuda()
    dc = N.DistanceCalculatorGpu()
    dc.SetQueries(qa)
    dc.SetDatabase(da)
    dc.SetReducedCodeMap(tmap)
    dc.SetSubsequenceLength(L)
    out = np.zeros(n, np.int8)
    d0 = torch.zeros(n, dtype=torch.int32, device="cuda")
    d1 = torch.zeros(n, dtype=torch.int32, device="cuda")
    dd = torch.zeros(n, dtype=torch.int8, device="cuda")
    dc.CalculateDistancesAsync(n, c0, c1, out, d0, d1, dd)
    torch.cuda.synchronize()
    exp = np.array([oracle.distance(params, a, int(x), b, int(y)) for x, y in
                    zip(c0[:5000], c1[:5000])], np.int8)
    assert np.array_equal(out[:5000], exp)


def test_set_query_seeds_expansion(torch_cuda):
    from gzb import native as N
    torch = torch_cuda
    rng = np.random.default_rng(3)
    nlist = 5000
    list_qid = rng.integers(0, 100, nlist).astype(np.uint32)
    list_qpos = rng.integers(0, 10**6, nlist).astype(np.uint32)
    runs = rng.integers(1, 40, 3000)
    seed_ids = rng.integers(0, nlist, len(runs)).astype(np.uint32)
    starts = np.concatenate([[0], np.cumsum(runs)[:-1]]).astype(np.uint32)
    size = int(runs.sum())
    u = N.UngappedExtenderGpu()
    tq = torch.from_numpy(list_qid).cuda()
    tp = torch.from_numpy(list_qpos).cuda()
    u.SetQuerySeedDataList(tq, tp)
    tb = N.UngappedExtenderGpu.QuerySeedsTempBytes(size)
    d_temp = torch.zeros(tb, dtype=torch.uint8, device="cuda")
    d_ids = torch.zeros(len(runs), dtype=torch.int32, device="cuda")
    d_starts = torch.zeros(len(runs), dtype=torch.int32, device="cuda")
    d_qid = torch.zeros(size, dtype=torch.int32, device="cuda")
    d_qp = torch.zeros(size, dtype=torch.int32, device="cuda")
    d_tmp = torch.zeros(size, dtype=torch.int32, device="cuda")
    u.SetQuerySeeds(len(runs), size, seed_ids, starts, tb, d_temp, d_ids, d_starts, d_qid,
                    d_qp, d_tmp)
    torch.cuda.synchronize()
    owner = np.repeat(seed_ids, runs)
    assert np.array_equal(d_qid.cpu().numpy().view(np.uint32), list_qid[owner])
    assert np.array_equal(d_qp.cpu().numpy().view(np.uint32), list_qpos[owner])


@pytest.mark.parametrize("group", [5, 6, 7, 8])
def test_gapped_group_kernels_match_oracle(torch_cuda, oracle, params, group):
    """GZB_GAPPED_KERNEL_GROUP4..32 (4..32 lanes per extension) through the
    operator API: every X-drop in both directions against the oracle (X-drops
    outside the group DP's exact range run the rows kernel), and long
    homologs whose bands outgrow the group's 64 columns."""
    from gzb import native as N
    keep = N.get_tile_parameter(N.TILE_GAPPED_KERNEL)
    N.set_tile_parameter(N.TILE_GAPPED_KERNEL, group)
    try:
        for cutoff in (0, 5, 26, 60, 2000, INT_MAX):
            for reverse in (False, True):
                rng = np.random.default_rng(3000 + group * 31 + cutoff % 89 + (5 if reverse else 0))
                n = 200 if cutoff not in (2000, INT_MAX) else 60
                A, B = _pairs(rng, n, hi=600 if cutoff < 1000 else 250)
                qc, qs = _concat(A, 25)
                dc, ds = _concat(B, 25)
                qpos = [qs[i] + int(rng.integers(0, len(A[i]))) for i in range(n)]
                dpos = [ds[i] + int(np.clip(qpos[i] - qs[i] + rng.integers(-4, 5), 0,
                                            len(B[i]) - 1)) for i in range(n)]
                s, q, d, cells = _gapped_gpu(torch_cuda, params, qc, dc, qpos, dpos, reverse,
                                             cutoff)
                total = 0
                for i in range(n):
                    es, eq, ed, ec = oracle.gapped_one_side(params, qc, qpos[i], dc, dpos[i],
                                                            reverse, cutoff)
                    total += ec
                    assert (int(s[i]), int(q[i]), int(d[i])) == \
                        (es, int(qpos[i]) + eq, int(dpos[i]) + ed), (group, cutoff, reverse, i)
                assert cells == total
        rng = np.random.default_rng(78)
        A, B = _pairs(rng, 24, lo=2000, hi=8000)
        qc, qs = _concat(A, 25)
        dc, ds = _concat(B, 25)
        qpos = [qs[i] + len(A[i]) // 2 for i in range(24)]
        dpos = [ds[i] + len(A[i]) // 2 for i in range(24)]
        cutoff = int(params["gapped_cutoff"])
        for rev in (False, True):
            s, q, d, _ = _gapped_gpu(torch_cuda, params, qc, dc, qpos, dpos, rev, cutoff)
            for i in range(24):
                es, eq, ed, _ = oracle.gapped_one_side(params, qc, qpos[i], dc, dpos[i], rev,
                                                       cutoff)
                assert (int(s[i]), int(q[i]), int(d[i])) == (es, int(qpos[i]) + eq,
                                                             int(dpos[i]) + ed)
    finally:
        N.set_tile_parameter(N.TILE_GAPPED_KERNEL, keep)


@pytest.mark.parametrize("band", [32, 128])
def test_rows_kernel_band_widths_match_oracle(torch_cuda, oracle, params, band):
    """GZB_TILE_BAND_WIDTH 32 and 128 on the rows kernel through the operator
    API: every X-drop in both directions against the oracle, the cell count
    included (a band outgrowing the lane's columns goes to the warp kernel,
    or to the serial kernel for X-drops outside the warp DP's range)."""
    from gzb import native as N
    keep_k = N.get_tile_parameter(N.TILE_GAPPED_KERNEL)
    keep_w = N.get_tile_parameter(N.TILE_BAND_WIDTH)
    N.set_tile_parameter(N.TILE_GAPPED_KERNEL, N.GAPPED_KERNEL_ROWS)
    N.set_tile_parameter(N.TILE_BAND_WIDTH, band)
    try:
        for cutoff in (0, 5, 26, 60, 2000, INT_MAX):
            for reverse in (False, True):
                rng = np.random.default_rng(4000 + band + cutoff % 97 + (7 if reverse else 0))
                n = 200 if cutoff not in (2000, INT_MAX) else 60
                A, B = _pairs(rng, n, hi=600 if cutoff < 1000 else 250)
                qc, qs = _concat(A, 25)
                dc, ds = _concat(B, 25)
                qpos = [qs[i] + int(rng.integers(0, len(A[i]))) for i in range(n)]
                dpos = [ds[i] + int(np.clip(qpos[i] - qs[i] + rng.integers(-4, 5), 0,
                                            len(B[i]) - 1)) for i in range(n)]
                s, q, d, cells = _gapped_gpu(torch_cuda, params, qc, dc, qpos, dpos, reverse,
                                             cutoff)
                total = 0
                for i in range(n):
                    es, eq, ed, ec = oracle.gapped_one_side(params, qc, qpos[i], dc, dpos[i],
                                                            reverse, cutoff)
                    total += ec
                    assert (int(s[i]), int(q[i]), int(d[i])) == \
                        (es, int(qpos[i]) + eq, int(dpos[i]) + ed), (band, cutoff, reverse, i)
                assert cells == total
    finally:
        N.set_tile_parameter(N.TILE_GAPPED_KERNEL, keep_k)
        N.set_tile_parameter(N.TILE_BAND_WIDTH, keep_w)

