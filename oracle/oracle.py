"""ctypes bindings of the CPU oracle (test infrastructure only).

``Oracle`` wraps liboracle.so (the C restatement in gz_oracle.c);
``Reference`` wraps _ref/libgzref.so (the reference's own units, present only
where it was built from the reference checkout).  Used by the tests, the
smoke check and the CPU-baseline leg of the benchmark, never by the engine.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libgzref.so")
# reference checkout the pin library and programs are compiled from
# (build-time only; unset where there is no checkout)
REF_ROOT = os.environ.get("GZ_REFERENCE_ROOT")

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)

RESULT_DTYPE = np.dtype([
    ("chunk_id", "<i4"), ("subject_id", "<i4"), ("score", "<i4"),
    ("hit_q", "<u4"), ("hit_d", "<u4"), ("start_q", "<u4"), ("start_d", "<u4"),
    ("end_q", "<u4"), ("end_d", "<u4"),
])
COUNTER_NAMES = ("distance_seeds", "ungapped_seeds", "ungapped_hits",
                 "chained_hits", "gapped_extensions", "gapped_cells")


def build(ref: bool = False) -> None:
    """Compile liboracle.so; with ref=True and GZ_REFERENCE_ROOT naming a
    reference checkout, also the reference's units (_ref/libgzref.so) and
    programs (_ref/ghostz, _ref/ghostz-gpu-host)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
    if ref and REF_ROOT and os.path.isdir(os.path.join(REF_ROOT, "src")):
        subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", "aln", "alngpu",
                               f"REF_ROOT={REF_ROOT}"])


def _p(a, t):
    return a.ctypes.data_as(t)


def _pp(params):
    return C.c_void_p(params.__array_interface__["data"][0]) if hasattr(params, "__array_interface__") else C.c_void_p(np.asarray(params).ctypes.data)


class _Params:
    """Keeps a contiguous copy of a PARAMS_DTYPE record alive."""

    def __init__(self, p):
        self.arr = np.array([p], dtype=p.dtype)

    @property
    def ptr(self):
        return C.c_void_p(self.arr.ctypes.data)


class Oracle:
    def __init__(self, path: str = LIB):
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        self.L = L
        L.gzo_hash.argtypes = [C.c_void_p, u8p, u32p, u32p]
        L.gzo_distance.argtypes = [C.c_void_p, u8p, C.c_uint32, u8p, C.c_uint32]
        L.gzo_ungapped_one_side.argtypes = [C.c_void_p, u8p, u8p, C.c_int, C.c_int]
        L.gzo_ungapped_with_trigger.argtypes = [C.c_void_p, u8p, C.c_uint32, u8p,
                                                C.c_uint32, C.c_int, C.c_int]
        L.gzo_gapped_one_side.argtypes = [C.c_void_p, u8p, u8p, C.c_int, C.c_int,
                                          i32p, i32p, i32p, C.POINTER(C.c_uint64)]
        L.gzo_gapped_one_side_edits.argtypes = [C.c_void_p, u8p, u8p, C.c_int, C.c_int,
                                                i32p, i32p, i32p, u8p, C.c_size_t,
                                                C.POINTER(C.c_size_t)]
        L.gzo_build_alignment.argtypes = [C.c_void_p, u8p, C.c_uint32, u8p, C.c_uint32,
                                          C.c_void_p]
        L.gzo_chain_filter.argtypes = [C.c_void_p, u8p, C.c_uint32, C.c_int, u8p,
                                       u32p, u32p, C.c_size_t]
        L.gzo_chain_filter.restype = C.c_size_t
        L.gzo_db_index_build.argtypes = [C.c_void_p, u8p, C.c_uint32]
        L.gzo_db_index_build.restype = C.c_void_p
        L.gzo_db_index_free.argtypes = [C.c_void_p]
        L.gzo_db_index_array.argtypes = [C.c_void_p, C.c_int, C.POINTER(u32p)]
        L.gzo_db_index_array.restype = C.c_size_t
        L.gzo_query_lists_build.argtypes = [C.c_void_p, u8p, u32p, u32p, C.c_uint32]
        L.gzo_query_lists_build.restype = C.c_void_p
        L.gzo_query_lists_free.argtypes = [C.c_void_p]
        L.gzo_query_lists_array.argtypes = [C.c_void_p, C.c_int, C.POINTER(u32p)]
        L.gzo_query_lists_array.restype = C.c_size_t
        L.gzo_presearch_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, u8p, u32p,
                                        u32p, C.c_uint32, i32p, i32p, u8p, C.c_uint32,
                                        u32p, C.c_uint32, C.c_uint32, C.c_uint32]
        L.gzo_presearch_run.restype = C.c_void_p
        L.gzo_presearch_free.argtypes = [C.c_void_p]
        L.gzo_add_results.argtypes = [C.c_void_p, u32p, C.c_uint32, C.c_uint32, C.c_void_p,
                                      C.c_size_t, C.c_void_p, C.c_size_t]
        L.gzo_add_results.restype = C.c_size_t
        L.gzo_presearch_results.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]
        L.gzo_presearch_results.restype = C.c_size_t
        L.gzo_presearch_counters.argtypes = [C.c_void_p, C.POINTER(C.c_uint64 * 6)]
        L.gzo_presearch_hits.argtypes = [C.c_void_p, C.POINTER(u32p), C.POINTER(u32p),
                                         C.POINTER(u32p)]
        L.gzo_presearch_hits.restype = C.c_size_t
        L.gzo_query_karlin.argtypes = [C.c_void_p, u8p, C.c_uint32, C.c_float, C.c_float,
                                       C.POINTER(C.c_float), C.POINTER(C.c_float),
                                       C.POINTER(C.c_float), i32p, i32p]
        L.gzo_seg_mask.argtypes = [C.c_char_p, C.c_uint32, C.c_char_p]
        L.gzo_translate_query_seg.argtypes = [C.c_char_p, C.c_uint32, C.c_uint8, u8p]
        L.gzo_translate_query_seg.restype = C.c_uint32
        L.gzo_ln_factorial6.argtypes = [C.c_uint32]
        L.gzo_search_space.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_float, C.c_float,
                                       C.c_double, C.c_double]
        L.gzo_search_space.restype = C.c_uint64
        L.gzo_evalue.argtypes = [C.c_int32, C.c_uint64, C.c_float, C.c_float]
        L.gzo_evalue.restype = C.c_double
        L.gzo_bit_score.argtypes = [C.c_int32, C.c_float, C.c_float]
        L.gzo_bit_score.restype = C.c_float
        L.gzo_translated_real_start.argtypes = [C.c_uint32, C.c_uint32]
        L.gzo_translated_real_start.restype = C.c_uint32
        L.gzo_translated_real_end.argtypes = [C.c_uint32, C.c_uint32]
        L.gzo_translated_real_end.restype = C.c_uint32
        L.gzo_protein_query_seg.argtypes = [C.c_char_p, C.c_uint32, C.c_uint8, u8p]
        L.gzo_ln_factorial6.restype = C.c_double
        L.gzo_translated_length.argtypes = [C.c_uint32]
        L.gzo_translated_length.restype = C.c_uint32
        L.gzo_translate_query.argtypes = [C.c_char_p, C.c_uint32, C.c_uint8, u8p]
        L.gzo_translate_query.restype = C.c_uint32

    # -- primitives ---------------------------------------------------------
    def hash(self, params, seq, pos=0):
        pr = _Params(params)
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        h = C.c_uint32()
        ln = C.c_uint32()
        r = self.L.gzo_hash(pr.ptr, C.cast(C.c_void_p(seq.ctypes.data + int(pos)), u8p),
                            C.byref(h), C.byref(ln))
        return r, h.value, ln.value

    def distance(self, params, seq0, c0, seq1, c1):
        pr = _Params(params)
        s0 = np.ascontiguousarray(seq0, dtype=np.uint8)
        s1 = np.ascontiguousarray(seq1, dtype=np.uint8)
        return self.L.gzo_distance(pr.ptr, _p(s0, u8p), int(c0), _p(s1, u8p), int(c1))

    def ungapped_one_side(self, params, seq0, p0, seq1, p1, reversed_, cutoff):
        pr = _Params(params)
        s0 = np.ascontiguousarray(seq0, dtype=np.uint8)
        s1 = np.ascontiguousarray(seq1, dtype=np.uint8)
        return self.L.gzo_ungapped_one_side(
            pr.ptr, C.cast(C.c_void_p(s0.ctypes.data + int(p0)), u8p),
            C.cast(C.c_void_p(s1.ctypes.data + int(p1)), u8p), int(reversed_), int(cutoff))

    def ungapped_with_trigger(self, params, query, qpos, db, dpos, cutoff, trigger):
        pr = _Params(params)
        q = np.ascontiguousarray(query, dtype=np.uint8)
        d = np.ascontiguousarray(db, dtype=np.uint8)
        return self.L.gzo_ungapped_with_trigger(pr.ptr, _p(q, u8p), int(qpos), _p(d, u8p),
                                                int(dpos), int(cutoff), int(trigger))

    def gapped_one_side(self, params, seq0, p0, seq1, p1, reversed_, cutoff):
        pr = _Params(params)
        s0 = np.ascontiguousarray(seq0, dtype=np.uint8)
        s1 = np.ascontiguousarray(seq1, dtype=np.uint8)
        b, q, d = C.c_int32(), C.c_int32(), C.c_int32()
        cells = C.c_uint64()
        self.L.gzo_gapped_one_side(
            pr.ptr, C.cast(C.c_void_p(s0.ctypes.data + int(p0)), u8p),
            C.cast(C.c_void_p(s1.ctypes.data + int(p1)), u8p), int(reversed_), int(cutoff),
            C.byref(b), C.byref(q), C.byref(d), C.byref(cells))
        return b.value, q.value, d.value, cells.value

    def gapped_one_side_edits(self, params, seq0, p0, seq1, p1, reversed_, cutoff):
        """(score, best pos0, best pos1, ops) of the traceback extension."""
        pr = _Params(params)
        s0 = np.ascontiguousarray(seq0, dtype=np.uint8)
        s1 = np.ascontiguousarray(seq1, dtype=np.uint8)
        b, q, d = C.c_int32(), C.c_int32(), C.c_int32()
        cap = 1 << 18
        ops = np.zeros(cap, np.uint8)
        n = C.c_size_t()
        rc = self.L.gzo_gapped_one_side_edits(
            pr.ptr, C.cast(C.c_void_p(s0.ctypes.data + int(p0)), u8p),
            C.cast(C.c_void_p(s1.ctypes.data + int(p1)), u8p), int(reversed_), int(cutoff),
            C.byref(b), C.byref(q), C.byref(d), _p(ops, u8p), cap, C.byref(n))
        assert rc == 0
        return b.value, q.value, d.value, ops[:n.value].copy()

    def build_alignment(self, params, query, hit_q, db, hit_d):
        """AlignerCommon::BuildResult statistics of one hit (concatenated
        coordinates): a dict with score, start_q, start_d, end_q, end_d,
        alignment_length, mismatches, gap_openings, gap_extensions."""
        pr = _Params(params)
        q = np.ascontiguousarray(query, dtype=np.uint8)
        d = np.ascontiguousarray(db, dtype=np.uint8)
        out = (C.c_uint32 * 9)()
        rc = self.L.gzo_build_alignment(pr.ptr, _p(q, u8p), int(hit_q), _p(d, u8p), int(hit_d),
                                        C.byref(out))
        assert rc == 0
        v = list(out)
        v[0] = C.c_int32(v[0]).value
        return dict(zip(("score", "start_q", "start_d", "end_q", "end_d", "alignment_length",
                         "mismatches", "gap_openings", "gap_extensions"), v))

    def query_karlin(self, params, seq, ungapped_bits=7.0, trigger_bits=22.0):
        """(lambda, K, H, ungapped cutoff, gapped trigger) of one whole query
        (delimiters included)."""
        pr = _Params(params)
        s = np.ascontiguousarray(seq, dtype=np.uint8)
        lam, k, h = C.c_float(), C.c_float(), C.c_float()
        cut, trig = np.zeros(1, np.int32), np.zeros(1, np.int32)
        self.L.gzo_query_karlin(pr.ptr, _p(s, u8p), len(s), ungapped_bits, trigger_bits,
                                C.byref(lam), C.byref(k), C.byref(h), _p(cut, i32p),
                                _p(trig, i32p))
        return lam.value, k.value, h.value, int(cut[0]), int(trig[0])

    def seg_mask(self, seq):
        """SEG-masked copy of a protein string (bytes), or None when it is
        shorter than the window."""
        seq = bytes(seq)
        out = C.create_string_buffer(max(len(seq), 1))
        rc = self.L.gzo_seg_mask(seq, len(seq), out)
        return None if rc else out.raw[:len(seq)]

    def protein_query_seg(self, letters, delimiter):
        """ProteinQuery codes (length + 2) of one protein with SEG on."""
        letters = bytes(letters)
        out = np.zeros(len(letters) + 2, np.uint8)
        self.L.gzo_protein_query_seg(letters, len(letters), int(delimiter), _p(out, u8p))
        return out

    # BLOSUM62 with gaps 11/1: the gapped parameters WriteOutput uses
    GAPPED = (0.267, 0.041, 1.9, -30.0)

    def hit_statistics(self, query_length, db_length, db_sequences, score, gapped=GAPPED):
        """(search space, E-value, normalized score) of a result."""
        lam, k, alpha, beta = gapped
        ss = self.L.gzo_search_space(query_length, db_length, db_sequences, lam, k, alpha, beta)
        return ss, self.L.gzo_evalue(score, ss, lam, k), self.L.gzo_bit_score(score, lam, k)

    def translated_real(self, position, dna_length):
        return (self.L.gzo_translated_real_start(position, dna_length),
                self.L.gzo_translated_real_end(position, dna_length))

    def translate_query_seg(self, dna, delimiter):
        """translate_query with the SEG filter on."""
        dna = bytes(dna)
        out = np.zeros(self.L.gzo_translated_length(len(dna)), np.uint8)
        n = self.L.gzo_translate_query_seg(dna, len(dna), int(delimiter), _p(out, u8p))
        assert n == len(out)
        return out

    def translate_query(self, dna, delimiter):
        """Translated query codes of one DNA read (bytes): the six frames in
        the reference's TranslatedDnaQuery layout, delimiters included."""
        dna = bytes(dna)
        out = np.zeros(self.L.gzo_translated_length(len(dna)), np.uint8)
        n = self.L.gzo_translate_query(dna, len(dna), int(delimiter), _p(out, u8p))
        assert n == len(out)
        return out

    def chain_filter(self, params, query, qlen, cutoff, db, hq, hd):
        pr = _Params(params)
        q = np.ascontiguousarray(query, dtype=np.uint8)
        d = np.ascontiguousarray(db, dtype=np.uint8)
        hq = np.array(hq, dtype=np.uint32)
        hd = np.array(hd, dtype=np.uint32)
        n = self.L.gzo_chain_filter(pr.ptr, _p(q, u8p), int(qlen), int(cutoff), _p(d, u8p),
                                    _p(hq, u32p), _p(hd, u32p), len(hq))
        return hq[:n].copy(), hd[:n].copy()

    # -- index / lists --------------------------------------------------------
    def db_index(self, params, db_codes):
        pr = _Params(params)
        d = np.ascontiguousarray(db_codes, dtype=np.uint8)
        h = self.L.gzo_db_index_build(pr.ptr, _p(d, u8p), len(d))
        out = {}
        names = ("nc_keys", "nc_offsets", "nc_values", "rep_keys", "rep_offsets",
                 "rep_cluster_ids", "rep_positions", "member_offsets", "member_positions")
        for i, nm in enumerate(names):
            ptr = u32p()
            n = self.L.gzo_db_index_array(C.c_void_p(h), i, C.byref(ptr))
            out[nm] = np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.uint32)
        self.L.gzo_db_index_free(C.c_void_p(h))
        return out

    def query_lists(self, params, queries):
        pr = _Params(params)
        h = self.L.gzo_query_lists_build(pr.ptr, _p(queries.codes, u8p),
                                         _p(queries.offsets, u32p),
                                         _p(queries.lengths, u32p), queries.number)
        out = {}
        for i, nm in enumerate(("hashes", "offsets", "check_counts", "query_ids", "positions")):
            ptr = u32p()
            n = self.L.gzo_query_lists_array(C.c_void_p(h), i, C.byref(ptr))
            out[nm] = np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.uint32)
        self.L.gzo_query_lists_free(C.c_void_p(h))
        return out

    def add_results(self, params, db, added, results):
        """One AddResults step (gzo_add_results): `added` (RESULT_DTYPE, every
        record's chunk_id set to the chunk being merged; subject ids are
        recomputed from db's offsets) merged into `results`; returns the
        new list."""
        pr = _Params(params)
        b = int(params["max_number_results"])
        a = np.ascontiguousarray(added, dtype=RESULT_DTYPE).copy()
        r = np.zeros(max(b, len(results)) + 1, dtype=RESULT_DTYPE)
        r[:len(results)] = results
        offs = np.ascontiguousarray(db.offsets, dtype=np.uint32)
        n = self.L.gzo_add_results(pr.ptr, _p(offs, u32p), db.number_sequences, len(db.codes),
                                   C.c_void_p(a.ctypes.data), len(a),
                                   C.c_void_p(r.ctypes.data), len(results))
        return r[:n].copy()

    # -- presearch --------------------------------------------------------------
    def presearch(self, params, db, queries, query_begin=0, query_end=None):
        """Returns (results per query as RESULT_DTYPE arrays, counters dict,
        ungapped survivors (qid, q, d))."""
        import time
        pr = _Params(params)
        dbc = np.ascontiguousarray(db.codes, dtype=np.uint8)
        idx = self.L.gzo_db_index_build(pr.ptr, _p(dbc, u8p), len(dbc))
        t0 = time.perf_counter()  # search time: query lists + presearch
        lists = self.L.gzo_query_lists_build(pr.ptr, _p(queries.codes, u8p),
                                             _p(queries.offsets, u32p),
                                             _p(queries.lengths, u32p), queries.number)
        if query_end is None:
            query_end = queries.number
        cut = np.ascontiguousarray(queries.cutoffs, dtype=np.int32)
        trig = np.ascontiguousarray(queries.triggers, dtype=np.int32)
        offs = np.ascontiguousarray(db.offsets, dtype=np.uint32)
        h = self.L.gzo_presearch_run(pr.ptr, C.c_void_p(idx), C.c_void_p(lists),
                                     _p(queries.codes, u8p), _p(queries.offsets, u32p),
                                     _p(queries.lengths, u32p), queries.number,
                                     _p(cut, i32p), _p(trig, i32p), _p(dbc, u8p), len(dbc),
                                     _p(offs, u32p), db.number_sequences,
                                     query_begin, query_end)
        search_seconds = time.perf_counter() - t0
        results = []
        for qi in range(queries.number):
            ptr = C.c_void_p()
            n = self.L.gzo_presearch_results(C.c_void_p(h), qi, C.byref(ptr))
            if n:
                buf = (C.c_char * (n * RESULT_DTYPE.itemsize)).from_address(ptr.value)
                results.append(np.frombuffer(bytes(buf), dtype=RESULT_DTYPE).copy())
            else:
                results.append(np.zeros(0, dtype=RESULT_DTYPE))
        cnt = (C.c_uint64 * 6)()
        self.L.gzo_presearch_counters(C.c_void_p(h), C.byref(cnt))
        counters = dict(zip(COUNTER_NAMES, [int(v) for v in cnt]))
        counters["search_seconds"] = search_seconds
        a, b, c = u32p(), u32p(), u32p()
        n = self.L.gzo_presearch_hits(C.c_void_p(h), C.byref(a), C.byref(b), C.byref(c))
        hits = tuple(np.ctypeslib.as_array(x, shape=(n,)).copy() if n else np.zeros(0, np.uint32)
                     for x in (a, b, c))
        self.L.gzo_presearch_free(C.c_void_p(h))
        self.L.gzo_query_lists_free(C.c_void_p(lists))
        self.L.gzo_db_index_free(C.c_void_p(idx))
        return results, counters, hits


class Reference:
    """The reference's own units (built from the reference checkout)."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        self.L = L
        L.gzr_hash.argtypes = [C.c_void_p, u8p, u32p, u32p]
        L.gzr_hash_many.argtypes = [C.c_void_p, u8p, C.c_uint32, i32p, u32p, u32p]
        L.gzr_distances.argtypes = [C.c_void_p, u8p, u8p, C.c_size_t, u32p, u32p,
                                    C.POINTER(C.c_int8)]
        L.gzr_ungapped_one_side.argtypes = [C.c_void_p, u8p, u8p, C.c_int, C.c_int]
        L.gzr_gapped_one_side.argtypes = [C.c_void_p, u8p, C.c_uint32, u8p, C.c_int,
                                          C.c_int, i32p, i32p, i32p]
        L.gzr_gapped_one_side_edits.argtypes = [C.c_void_p, u8p, C.c_uint32, u8p, C.c_int,
                                                C.c_int, i32p, i32p, i32p, u8p, C.c_size_t,
                                                C.POINTER(C.c_size_t)]
        L.gzr_chain_filter.argtypes = [C.c_void_p, u8p, C.c_uint32, C.c_int, u8p, u32p,
                                       u32p, C.c_size_t]
        L.gzr_chain_filter.restype = C.c_size_t
        L.gzr_db_index_build.argtypes = [C.c_void_p, u8p, C.c_uint32]
        L.gzr_db_index_build.restype = C.c_void_p
        L.gzr_db_index_free.argtypes = [C.c_void_p]
        L.gzr_db_index_lookup.argtypes = [C.c_void_p, C.c_int, C.c_uint32, u32p, C.c_size_t]
        L.gzr_db_index_lookup.restype = C.c_size_t
        L.gzr_db_index_members.argtypes = [C.c_void_p, C.c_uint32, u32p, C.c_size_t]
        L.gzr_db_index_members.restype = C.c_size_t
        L.gzr_db_index_max_mismatches.argtypes = [C.c_void_p]
        L.gzr_db_index_save.argtypes = [C.c_void_p, u8p, C.c_size_t]
        L.gzr_db_index_save.restype = C.c_size_t
        L.gzr_db_index_save_common.argtypes = [C.c_void_p, u8p, C.c_size_t]
        L.gzr_db_index_save_common.restype = C.c_size_t
        L.gzr_ungapped_karlin.argtypes = [C.c_void_p, u8p, C.c_uint32, C.POINTER(C.c_float),
                                          C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.gzr_normalized_cutoff_to_nominal.argtypes = [C.c_float, C.c_float, C.c_float]
        L.gzr_normalized_to_nominal.argtypes = [C.c_float, C.c_float, C.c_float]
        L.gzr_translate_query.argtypes = [C.c_void_p, C.c_char_p, C.c_uint32, u8p, C.c_uint32]
        L.gzr_translate_query.restype = C.c_uint32
        L.gzr_seg_mask.argtypes = [C.c_char_p, C.c_uint32, C.c_char_p]
        L.gzr_translate_query_seg.argtypes = [C.c_void_p, C.c_char_p, C.c_uint32, u8p,
                                              C.c_uint32]
        L.gzr_translate_query_seg.restype = C.c_uint32
        L.gzr_hit_statistics.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64,
                                         C.c_int32, C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_double), C.POINTER(C.c_float)]
        L.gzr_translated_real.argtypes = [C.c_void_p, C.c_char_p, C.c_uint32, C.c_uint32,
                                          u32p, u32p]
        L.gzr_protein_query_seg.argtypes = [C.c_void_p, C.c_char_p, C.c_uint32, u8p,
                                            C.c_uint32, C.POINTER(C.c_float),
                                            C.POINTER(C.c_float)]
        L.gzr_protein_query_seg.restype = C.c_uint32

    def hash_many(self, params, seq):
        pr = _Params(params)
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        n = len(seq) - 8
        r = np.zeros(n, np.int32)
        h = np.zeros(n, np.uint32)
        ln = np.zeros(n, np.uint32)
        self.L.gzr_hash_many(pr.ptr, _p(seq, u8p), n, _p(r, i32p), _p(h, u32p), _p(ln, u32p))
        return r, h, ln

    def distances(self, params, seq0, seq1, c0, c1):
        pr = _Params(params)
        s0 = np.ascontiguousarray(seq0, dtype=np.uint8)
        s1 = np.ascontiguousarray(seq1, dtype=np.uint8)
        c0 = np.ascontiguousarray(c0, dtype=np.uint32)
        c1 = np.ascontiguousarray(c1, dtype=np.uint32)
        out = np.zeros(len(c0), np.int8)
        self.L.gzr_distances(pr.ptr, _p(s0, u8p), _p(s1, u8p), len(c0), _p(c0, u32p),
                             _p(c1, u32p), out.ctypes.data_as(C.POINTER(C.c_int8)))
        return out

    def ungapped_one_side(self, params, seq0, p0, seq1, p1, reversed_, cutoff):
        pr = _Params(params)
        s0 = np.ascontiguousarray(seq0, dtype=np.uint8)
        s1 = np.ascontiguousarray(seq1, dtype=np.uint8)
        return self.L.gzr_ungapped_one_side(
            pr.ptr, C.cast(C.c_void_p(s0.ctypes.data + int(p0)), u8p),
            C.cast(C.c_void_p(s1.ctypes.data + int(p1)), u8p), int(reversed_), int(cutoff))

    def gapped_one_side(self, params, seq0, p0, len0, seq1, p1, reversed_, cutoff):
        pr = _Params(params)
        s0 = np.ascontiguousarray(seq0, dtype=np.uint8)
        s1 = np.ascontiguousarray(seq1, dtype=np.uint8)
        b, q, d = C.c_int32(), C.c_int32(), C.c_int32()
        self.L.gzr_gapped_one_side(
            pr.ptr, C.cast(C.c_void_p(s0.ctypes.data + int(p0)), u8p), len0,
            C.cast(C.c_void_p(s1.ctypes.data + int(p1)), u8p), int(reversed_), int(cutoff),
            C.byref(b), C.byref(q), C.byref(d))
        return b.value, q.value, d.value

    def gapped_one_side_edits(self, params, seq0, p0, len0, seq1, p1, reversed_, cutoff):
        pr = _Params(params)
        s0 = np.ascontiguousarray(seq0, dtype=np.uint8)
        s1 = np.ascontiguousarray(seq1, dtype=np.uint8)
        b, q, d = C.c_int32(), C.c_int32(), C.c_int32()
        cap = 1 << 18
        ops = np.zeros(cap, np.uint8)
        n = C.c_size_t()
        rc = self.L.gzr_gapped_one_side_edits(
            pr.ptr, C.cast(C.c_void_p(s0.ctypes.data + int(p0)), u8p), len0,
            C.cast(C.c_void_p(s1.ctypes.data + int(p1)), u8p), int(reversed_), int(cutoff),
            C.byref(b), C.byref(q), C.byref(d), _p(ops, u8p), cap, C.byref(n))
        assert rc == 0
        return b.value, q.value, d.value, ops[:n.value].copy()

    def chain_filter(self, params, query, qlen, cutoff, db, hq, hd):
        pr = _Params(params)
        q = np.ascontiguousarray(query, dtype=np.uint8)
        d = np.ascontiguousarray(db, dtype=np.uint8)
        hq = np.array(hq, dtype=np.uint32)
        hd = np.array(hd, dtype=np.uint32)
        n = self.L.gzr_chain_filter(pr.ptr, _p(q, u8p), qlen, int(cutoff), _p(d, u8p),
                                    _p(hq, u32p), _p(hd, u32p), len(hq))
        return hq[:n].copy(), hd[:n].copy()

    def db_index(self, params, db_codes):
        pr = _Params(params)
        d = np.ascontiguousarray(db_codes, dtype=np.uint8)
        self._keep = d
        return self.L.gzr_db_index_build(pr.ptr, _p(d, u8p), len(d))

    def lookup(self, h, which, key, cap=1 << 22):
        out = np.zeros(cap, np.uint32)
        n = self.L.gzr_db_index_lookup(C.c_void_p(h), which, key, _p(out, u32p), cap)
        return out[: (2 * n if which == 1 else n)].copy()

    def members(self, h, cid, cap=1 << 22):
        out = np.zeros(cap, np.uint32)
        n = self.L.gzr_db_index_members(C.c_void_p(h), cid, _p(out, u32p), cap)
        return out[:n].copy()

    def save_index(self, h):
        """The bytes of the chunk's .sdp file the reference writes for h."""
        n = self.L.gzr_db_index_save(C.c_void_p(h), None, 0)
        out = np.zeros(n, np.uint8)
        self.L.gzr_db_index_save(C.c_void_p(h), _p(out, u8p), n)
        return out

    def save_common(self, h):
        """The bytes of the database's .scp file the reference writes for h."""
        n = self.L.gzr_db_index_save_common(C.c_void_p(h), None, 0)
        out = np.zeros(n, np.uint8)
        self.L.gzr_db_index_save_common(C.c_void_p(h), _p(out, u8p), n)
        return out

    def free_index(self, h):
        self.L.gzr_db_index_free(C.c_void_p(h))

    def ungapped_karlin(self, params, seq_with_delims):
        pr = _Params(params)
        s = np.ascontiguousarray(seq_with_delims, dtype=np.uint8)
        lam, k, h = C.c_float(), C.c_float(), C.c_float()
        self.L.gzr_ungapped_karlin(pr.ptr, _p(s, u8p), len(s), C.byref(lam), C.byref(k),
                                   C.byref(h))
        return lam.value, k.value, h.value

    def cutoffs(self, lam, k, ungapped_bits=7.0, trigger_bits=22.0):
        return (self.L.gzr_normalized_cutoff_to_nominal(ungapped_bits, lam, k),
                self.L.gzr_normalized_to_nominal(trigger_bits, lam, k))

    def translate_query(self, params, dna):
        """The reference's TranslatedDnaQuery codes of one DNA read (bytes,
        at least 3 bases)."""
        pr = _Params(params)
        dna = bytes(dna)
        assert len(dna) >= 3
        cap = 7 + 6 * (len(dna) // 3)
        out = np.zeros(cap, np.uint8)
        n = self.L.gzr_translate_query(pr.ptr, dna, len(dna), _p(out, u8p), cap)
        assert n == cap
        return out

    def seg_mask(self, seq):
        seq = bytes(seq)
        out = C.create_string_buffer(max(len(seq), 1))
        rc = self.L.gzr_seg_mask(seq, len(seq), out)
        return None if rc else out.raw[:len(seq)]

    def translate_query_seg(self, params, dna):
        pr = _Params(params)
        dna = bytes(dna)
        assert len(dna) >= 3
        cap = 7 + 6 * (len(dna) // 3)
        out = np.zeros(cap, np.uint8)
        n = self.L.gzr_translate_query_seg(pr.ptr, dna, len(dna), _p(out, u8p), cap)
        assert n == cap
        return out

    def protein_query_seg(self, params, letters):
        """(codes, lambda, K) of the reference's ProteinQuery with SEG on."""
        pr = _Params(params)
        letters = bytes(letters)
        out = np.zeros(len(letters) + 2, np.uint8)
        lam, k = C.c_float(), C.c_float()
        n = self.L.gzr_protein_query_seg(pr.ptr, letters, len(letters), _p(out, u8p),
                                         len(out), C.byref(lam), C.byref(k))
        assert n == len(out)
        return out, lam.value, k.value

    def hit_statistics(self, params, query_length, db_length, db_sequences, score):
        pr = _Params(params)
        ss, ev, bs = C.c_uint64(), C.c_double(), C.c_float()
        rc = self.L.gzr_hit_statistics(pr.ptr, query_length, db_length, db_sequences, score,
                                       C.byref(ss), C.byref(ev), C.byref(bs))
        assert rc == 0
        return ss.value, ev.value, bs.value

    def translated_real(self, params, dna, position):
        pr = _Params(params)
        dna = bytes(dna)
        st, en = np.zeros(1, np.uint32), np.zeros(1, np.uint32)
        self.L.gzr_translated_real(pr.ptr, dna, len(dna), position, _p(st, u32p), _p(en, u32p))
        return int(st[0]), int(en[0])
