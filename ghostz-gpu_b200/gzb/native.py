"""ctypes bindings of libghostz_b200.so.

The operator classes mirror the reference's GPU operator classes
(DistanceCalculatorGpu, UngappedExtenderGpu, GappedExtenderGpu) method for
method; device buffers are passed as integer device addresses (for example
``tensor.data_ptr()`` of a CUDA torch tensor) and host buffers as numpy
arrays.  Every call raises GzbError when the library reports a failure.
The library must exist: nothing here falls back to a CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import LIB

_lib = None


class GzbError(RuntimeError):
    pass


def symbols_declared_in_header():
    """Names of every function the public header declares."""
    import re
    hdr = os.path.join(os.path.dirname(os.path.dirname(LIB)), "include", "ghostz_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(gzb_[a-z0-9_]+)\s*\(", text)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise GzbError(f"{LIB} is missing: build it with gzb.build.build()")
        _lib = C.CDLL(LIB)
        _declare(_lib)
    return _lib


V = C.c_void_p
SZ = C.c_size_t
U32 = C.c_uint32
I32 = C.c_int32


def _declare(L):
    L.gzb_last_error.restype = C.c_char_p
    L.gzb_error_string.restype = C.c_char_p
    L.gzb_ungapped_extender_query_seeds_temp_bytes.restype = SZ
    L.gzb_ungapped_extender_query_seeds_temp_bytes.argtypes = [SZ]
    L.gzb_cost_model_param_count.restype = C.c_int
    L.gzb_cost_model_param_count.argtypes = []
    L.gzb_translated_query_length.restype = C.c_uint64
    L.gzb_translated_query_length.argtypes = [U32]
    L.gzb_gapped_karlin_parameters.argtypes = [C.c_char_p, C.c_int, C.c_int] + [V] * 5
    L.gzb_gapped_karlin_parameters.restype = C.c_int
    L.gzb_search_space.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_float, C.c_float,
                                   C.c_double, C.c_double]
    L.gzb_search_space.restype = C.c_uint64
    L.gzb_evalue.argtypes = [C.c_int32, C.c_uint64, C.c_float, C.c_float]
    L.gzb_evalue.restype = C.c_double
    L.gzb_bit_score.argtypes = [C.c_int32, C.c_float, C.c_float]
    L.gzb_bit_score.restype = C.c_float
    L.gzb_translated_real_start.argtypes = [U32, U32]
    L.gzb_translated_real_start.restype = U32
    L.gzb_translated_real_end.argtypes = [U32, U32]
    L.gzb_translated_real_end.restype = U32
    sigs = {
        "gzb_distance_calculator_create": [V],
        "gzb_distance_calculator_destroy": [V],
        "gzb_distance_calculator_set_queries": [V, V],
        "gzb_distance_calculator_set_database": [V, V],
        "gzb_distance_calculator_set_reduced_code_map": [V, V],
        "gzb_distance_calculator_set_subsequence_length": [V, U32],
        "gzb_distance_calculator_calculate_distances_async": [V, SZ, V, V, V, V, V, V, V],
        "gzb_ungapped_extender_create": [V],
        "gzb_ungapped_extender_destroy": [V],
        "gzb_ungapped_extender_set_query_seed_data_list": [V, V, V],
        "gzb_ungapped_extender_set_queries": [V, C.c_uint8, V, V, V],
        "gzb_ungapped_extender_set_database": [V, V],
        "gzb_ungapped_extender_set_score_matrix": [V, V, U32],
        "gzb_ungapped_extender_set_query_seeds": [V, SZ, SZ, V, V, SZ, V, V, V, V, V, V, V],
        "gzb_ungapped_extender_extend_with_trigger_async": [V, SZ, V, V, V, V, V, V, V, V, V, V],
        "gzb_gapped_extender_create": [V],
        "gzb_gapped_extender_destroy": [V],
        "gzb_gapped_extender_set_queries": [V, C.c_uint8, V],
        "gzb_gapped_extender_set_database": [V, V],
        "gzb_gapped_extender_set_score_parameters": [V, V, U32, C.c_int, C.c_int, C.c_int],
        "gzb_gapped_extender_convert_to_gapped_extension_seeds_async": [V, SZ, C.c_int, V, V, V, V, V, V, V, V],
        "gzb_gapped_extender_extend_one_side_score_only_async": [V, SZ, C.c_int, V, V, V, V, V, V, V],
        "gzb_gapped_extender_cells": [V, V],
        "gzb_gapped_extend_one_side_score_only_noalloc": [V, V, C.c_uint8, V, U32, C.c_int,
                                                          C.c_int, C.c_int, SZ, C.c_int, V, V,
                                                          V, V],
        "gzb_engine_create": [C.c_int, V],
        "gzb_engine_destroy": [V],
        "gzb_engine_set_params": [V, V],
        "gzb_engine_set_database": [V, I32, V, C.c_uint64, V, U32, V],
        "gzb_engine_set_queries": [V, V, C.c_uint64, V, V, U32, V, V, V],
        "gzb_engine_set_protein_queries": [V, V, C.c_uint64, V, V, U32, C.c_int, C.c_float,
                                           C.c_float, V, V, V],
        "gzb_engine_set_translated_queries": [V, V, V, U32, C.c_int, C.c_float, C.c_float, V,
                                              V, V],
        "gzb_engine_presearch": [V, C.c_int, V],
        "gzb_engine_reset_results": [V, V],
        "gzb_engine_get_results": [V, V, V, V],
        "gzb_engine_get_counters": [V, V],
        "gzb_engine_get_hits": [V, V, V, V, C.c_uint64, V, V],
        "gzb_engine_get_index_array": [V, C.c_int, V, C.c_uint64, V, V],
        "gzb_engine_get_list_array": [V, C.c_int, V, C.c_uint64, V, V],
        "gzb_engine_get_stage_ms": [V, V],
        "gzb_cost_model_init": [V, C.c_uint64],
        "gzb_cost_model_gradients": [V, V, V, U32, V, V, V],
        "gzb_cost_model_predict": [V, V, U32, V, V],
        "gzb_cost_model_train": [V, V, U32, V, C.c_int, C.c_int, C.c_float, C.c_uint64, V, V],
        "gzb_engine_set_logging": [V, C.c_int, C.c_uint64],
        "gzb_engine_get_log": [V, V, V, C.c_uint64, V],
        "gzb_engine_train_cost_model": [V, C.c_int, C.c_int, C.c_float, C.c_uint64, V, V],
        "gzb_engine_set_cost_model": [V, V],
        "gzb_engine_get_schedule_stats": [V, V, V],
        "gzb_set_tile_parameter": [C.c_int, C.c_int],
        "gzb_get_tile_parameter": [C.c_int, V],
        "gzb_engine_autotune": [V, C.c_int, C.c_int, V, C.c_int, V, V, V],
        "gzb_engine_set_tile": [V, C.c_int, C.c_int, C.c_int],
        "gzb_engine_get_tile": [V, C.c_int, C.c_int, V],
        "gzb_engine_get_extension_costs": [V, V, V, C.c_uint64, V, V],
        "gzb_engine_build_alignments": [V, V, V, V],
        "gzb_engine_index_bytes": [V, V],
        "gzb_engine_export_index": [V, V, C.c_uint64, V],
        "gzb_engine_set_database_with_index": [V, C.c_int32, V, C.c_uint64, V, C.c_uint32, V,
                                               C.c_uint64, V],
        "gzb_translate_dna_queries": [V, V, V, U32, V, C.c_uint8, V, V],
        "gzb_engine_swap_database": [V, U32, V],
        "gzb_engine_set_graph": [V, C.c_int],
        "gzb_engine_reserve": [V, C.c_uint64, C.c_uint64],
        "gzb_engine_get_graph_stats": [V, V, V, V],
        "gzb_engine_prefetch_database_with_index": [V, U32, C.c_int32, V, C.c_uint64, V, U32,
                                                    V, C.c_uint64, V],
        "gzb_query_karlin_cutoffs": [V, V, V, U32, V, U32, C.c_float, C.c_float, V, V, V, V],
        "gzb_seg_translated_queries": [V, V, V, U32, V, V],
        "gzb_seg_protein_queries": [V, V, V, U32, V, V],
        "gzb_index_blob_from_reference": [V, V, C.c_uint64, V, C.c_uint64, V, U32, V,
                                          C.c_uint64, V],
        "gzb_merge_chunk_results": [V, U32, V, V, V, V],
        "gzb_params_from_reference_common": [V, C.c_uint64, V],
        "gzb_sort_alignments": [U32, U32, V, V, U32, V, V],
        "gzb_write_hit_table": [U32, U32, V, V, V, V, U32, V, C.c_uint64, C.c_uint64, V, V,
                                C.c_float, C.c_float, C.c_double, C.c_double, V, C.c_uint64, V],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int


def check(rc):
    if rc != 0:
        L = lib()
        raise GzbError(f"{L.gzb_error_string(rc).decode()}: {L.gzb_last_error().decode()}")


def hptr(a):
    """Host pointer of a numpy array (None -> NULL)."""
    return None if a is None else C.c_void_p(a.ctypes.data)


def dptr(x):
    """Device pointer of a torch tensor / int address (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, int):
        return C.c_void_p(x)
    return C.c_void_p(x.data_ptr())


def stream_handle(stream=None):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


class _Handle:
    _kind = ""

    def __init__(self):
        h = C.c_void_p()
        check(getattr(lib(), f"gzb_{self._kind}_create")(C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            getattr(lib(), f"gzb_{self._kind}_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, name, *args):
        check(getattr(lib(), f"gzb_{self._kind}_{name}")(self.h, *args))


class DistanceCalculatorGpu(_Handle):
    """src/distance_calculator_gpu.h:18-40"""
    _kind = "distance_calculator"

    def SetQueries(self, d_queries):
        self._call("set_queries", dptr(d_queries))

    def SetDatabase(self, d_db):
        self._call("set_database", dptr(d_db))

    def SetReducedCodeMap(self, d_map):
        self._call("set_reduced_code_map", dptr(d_map))

    def SetSubsequenceLength(self, length):
        self._call("set_subsequence_length", int(length))

    def CalculateDistancesAsync(self, size, h_q, h_d, h_out, d_q, d_d, d_out, stream=None):
        self._call("calculate_distances_async", size, hptr(h_q), hptr(h_d), hptr(h_out),
                   dptr(d_q), dptr(d_d), dptr(d_out), stream_handle(stream))


class UngappedExtenderGpu(_Handle):
    """src/ungapped_extender_gpu.h:21-76"""
    _kind = "ungapped_extender"

    def SetQuerySeedDataList(self, d_query_ids, d_query_positions):
        self._call("set_query_seed_data_list", dptr(d_query_ids), dptr(d_query_positions))

    def SetQueries(self, delimiter, d_queries, d_cutoffs, d_triggers):
        self._call("set_queries", int(delimiter), dptr(d_queries), dptr(d_cutoffs),
                   dptr(d_triggers))

    def SetDatabase(self, d_db):
        self._call("set_database", dptr(d_db))

    def SetScoreMatrix(self, d_matrix, number_letters):
        self._call("set_score_matrix", dptr(d_matrix), int(number_letters))

    @staticmethod
    def QuerySeedsTempBytes(size):
        return int(lib().gzb_ungapped_extender_query_seeds_temp_bytes(size))

    def SetQuerySeeds(self, query_seeds_size, size, h_seed_ids, h_seed_starts, temp_bytes,
                      d_temp, d_seed_ids, d_seed_starts, d_query_ids, d_qpos, d_temp_array,
                      stream=None):
        self._call("set_query_seeds", query_seeds_size, size, hptr(h_seed_ids),
                   hptr(h_seed_starts), temp_bytes, dptr(d_temp), dptr(d_seed_ids),
                   dptr(d_seed_starts), dptr(d_query_ids), dptr(d_qpos), dptr(d_temp_array),
                   stream_handle(stream))

    def ExtendWithTriggerAsync(self, size, h_qid, h_qpos, h_dpos, h_flags, d_qid, d_qpos,
                               d_dpos, d_flags, d_temp=None, stream=None):
        self._call("extend_with_trigger_async", size, hptr(h_qid), hptr(h_qpos),
                   hptr(h_dpos), hptr(h_flags), dptr(d_qid), dptr(d_qpos), dptr(d_dpos),
                   dptr(d_flags), dptr(d_temp), stream_handle(stream))


class GappedExtenderGpu(_Handle):
    """src/gapped_extender_gpu.h:19-60"""
    _kind = "gapped_extender"

    def SetQueries(self, delimiter, d_queries):
        self._call("set_queries", int(delimiter), dptr(d_queries))

    def SetDatabase(self, d_db):
        self._call("set_database", dptr(d_db))

    def SetScoreParameters(self, d_matrix, number_letters, gap_open, gap_ext, cutoff):
        self._call("set_score_parameters", dptr(d_matrix), int(number_letters),
                   int(gap_open), int(gap_ext), int(cutoff))

    def ConvertToGappedExtensionSeedsAsync(self, size, reverse, h_seed_pos, h_qpos, h_dpos,
                                           d_seed_pos, d_temp, d_qpos, d_dpos, stream=None):
        self._call("convert_to_gapped_extension_seeds_async", size, int(bool(reverse)),
                   hptr(h_seed_pos), hptr(h_qpos), hptr(h_dpos), dptr(d_seed_pos),
                   dptr(d_temp), dptr(d_qpos), dptr(d_dpos), stream_handle(stream))

    def ExtendOneSideScoreOnlyAsync(self, size, reverse, h_qpos, h_dpos, h_scores, d_qpos,
                                    d_dpos, d_scores, stream=None):
        self._call("extend_one_side_score_only_async", size, int(bool(reverse)),
                   hptr(h_qpos), hptr(h_dpos), hptr(h_scores), dptr(d_qpos), dptr(d_dpos),
                   dptr(d_scores), stream_handle(stream))

    def Cells(self):
        c = C.c_uint64()
        self._call("cells", C.byref(c))
        return c.value


PAD = 256  # readable bytes kept before and after every device sequence


def device_sequence(codes, delimiter, device="cuda"):
    """Uploads codes with PAD delimiter bytes on both sides; returns
    (tensor, address of codes[0])."""
    import torch
    buf = np.full(len(codes) + 2 * PAD, delimiter, dtype=np.uint8)
    buf[PAD:PAD + len(codes)] = codes
    t = torch.from_numpy(buf).to(device)
    return t, t.data_ptr() + PAD


def device_matrix(matrix, device="cuda"):
    """(n+1)^2 int32 with zero delimiter row/column (the reference's device
    layout, src/aligner_gpu_data.cu:108-122)."""
    import torch
    m = np.asarray(matrix, dtype=np.int32)
    n = m.shape[0]
    out = np.zeros((n + 1, n + 1), dtype=np.int32)
    out[:n, :n] = m
    return torch.from_numpy(out.reshape(-1).copy()).to(device)


RESULT_DTYPE = np.dtype([
    ("chunk_id", "<i4"), ("subject_id", "<i4"), ("score", "<i4"),
    ("hit_q", "<u4"), ("hit_d", "<u4"), ("start_q", "<u4"), ("start_d", "<u4"),
    ("end_q", "<u4"), ("end_d", "<u4"),
])
ALIGNMENT_DTYPE = np.dtype([
    ("chunk_id", "<i4"), ("subject_id", "<i4"), ("score", "<i4"),
    ("hit_q", "<u4"), ("hit_d", "<u4"), ("start_q", "<u4"), ("start_d", "<u4"),
    ("end_q", "<u4"), ("end_d", "<u4"), ("alignment_length", "<u4"), ("mismatches", "<u4"),
    ("gap_openings", "<u4"), ("gap_extensions", "<u4"), ("presearch_score", "<i4"),
])
COUNTER_NAMES = ("distance_seeds", "ungapped_seeds", "ungapped_hits",
                 "chained_hits", "gapped_extensions", "gapped_cells", "gapped_fallbacks",
                 "ungapped_steps", "kernel_launches")
LIST_NAMES = ("hashes", "offsets", "check_counts", "query_ids", "positions")
INDEX_NAMES = ("nc_keys", "nc_offsets", "nc_values", "rep_keys", "rep_offsets",
               "rep_cluster_ids", "rep_positions", "member_offsets", "member_positions")
SCHEDULE_PLAIN = 0
SCHEDULE_BATCHED = 1
SCHEDULE_ORACLE = 2
TILE_BOOK_THRESHOLD = 0
TILE_GAPPED_KERNEL = 1
TILE_ORDER = 2
TILE_SEED_WALKER = 3
SEED_WALKER_UNIT = 0
SEED_WALKER_DEALT = 1
TILE_BAND_WIDTH = 4        # the rows kernel's band columns per lane: 32, 64, 128
ORDER_HITS = 0
ORDER_MODEL = 1
GAPPED_KERNEL_FLAT = 0
GAPPED_KERNEL_LANE = 1
GAPPED_KERNEL_ROWS = 2
GAPPED_KERNEL_STATIC = 3
GAPPED_KERNEL_DEAL = 4
GAPPED_KERNEL_GROUP4 = 5
GAPPED_KERNEL_GROUP8 = 6
GAPPED_KERNEL_GROUP16 = 7
GAPPED_KERNEL_GROUP32 = 8
COST_FEATURES = 8


def set_tile_parameter(which, value):
    """Process-wide default of tile parameter `which` (the operators' and
    engines' without a tuned tile)."""
    check(lib().gzb_set_tile_parameter(int(which), int(value)))


def get_tile_parameter(which):
    v = C.c_int()
    check(lib().gzb_get_tile_parameter(int(which), C.byref(v)))
    return int(v.value)


def cost_param_count():
    return int(lib().gzb_cost_model_param_count())


def cost_model_init(seed=0):
    p = np.zeros(cost_param_count(), np.float32)
    check(lib().gzb_cost_model_init(hptr(p), int(seed)))
    return p


class PresearchEngine:
    """Device-resident presearch of one database chunk at a time: the seed
    search, distance filter, ungapped and gapped extension and top-b merge
    that AlignerGpuPresearchThread::Run drives
    (src/aligner_gpu_presearch_thread.cpp:62-642)."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        check(lib().gzb_engine_create(int(device), C.byref(self.h)))
        self.params = None
        self.number_queries = 0

    def close(self):
        if self.h:
            lib().gzb_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        self.params = np.array([params], dtype=params.dtype)
        check(lib().gzb_engine_set_params(self.h, C.c_void_p(self.params.ctypes.data)))

    def set_database(self, db, chunk_id=0, stream=None, index=None):
        """Uploads a chunk and builds its device index, or takes the index
        from `index`, a blob export_index() wrote for the same chunk."""
        codes = np.ascontiguousarray(db.codes, dtype=np.uint8)
        offs = np.ascontiguousarray(db.offsets, dtype=np.uint32)
        if index is None:
            check(lib().gzb_engine_set_database(self.h, int(chunk_id), hptr(codes), len(codes),
                                                hptr(offs), int(db.number_sequences),
                                                _stream_or_null(stream)))
        else:
            blob = np.ascontiguousarray(index, dtype=np.uint8)
            check(lib().gzb_engine_set_database_with_index(
                self.h, int(chunk_id), hptr(codes), len(codes), hptr(offs),
                int(db.number_sequences), hptr(blob), blob.nbytes, _stream_or_null(stream)))

    def set_graph(self, enable=True):
        """Graph mode: the presearch runs as one captured CUDA graph."""
        check(lib().gzb_engine_set_graph(self.h, 1 if enable else 0))

    def reserve(self, hits, member_work):
        """Capacities of the hit and member-work buffers (graph mode)."""
        check(lib().gzb_engine_reserve(self.h, int(hits), int(member_work)))

    def graph_stats(self):
        """(captures, graph runs, eager redos) of graph mode."""
        v = [C.c_uint64() for _ in range(3)]
        check(lib().gzb_engine_get_graph_stats(self.h, *[C.byref(x) for x in v]))
        return tuple(int(x.value) for x in v)

    def swap_database(self, slot, stream=None):
        """Exchanges the resident chunk with the chunk stored in `slot`."""
        check(lib().gzb_engine_swap_database(self.h, int(slot), _stream_or_null(stream)))

    def prefetch_database(self, slot, db, blob, chunk_id=0, stream=None):
        """Fills `slot` from host arrays and an index blob with asynchronous
        copies on `stream` (numpy arrays; pass pinned memory for overlap).
        The arrays must stay alive until the slot is swapped in."""
        codes = np.ascontiguousarray(db.codes, dtype=np.uint8)
        offs = np.ascontiguousarray(db.offsets, dtype=np.uint32)
        check(lib().gzb_engine_prefetch_database_with_index(
            self.h, int(slot), int(chunk_id), hptr(codes), len(codes), hptr(offs),
            int(db.number_sequences), hptr(blob), blob.nbytes, _stream_or_null(stream)))
        self._pinned_refs = getattr(self, "_pinned_refs", {})
        self._pinned_refs[int(slot)] = (codes, offs, blob)

    def index_bytes(self):
        """Bytes of the resident chunk's index blob."""
        n = C.c_uint64()
        check(lib().gzb_engine_index_bytes(self.h, C.byref(n)))
        return int(n.value)

    def export_index(self, stream=None, out=None):
        """The resident chunk's device index as a host blob (numpy uint8),
        written into `out` (a uint8 array of index_bytes(), pinned memory
        for example) when given."""
        n = self.index_bytes()
        blob = np.zeros(n, np.uint8) if out is None else out
        assert blob.dtype == np.uint8 and blob.nbytes >= n
        check(lib().gzb_engine_export_index(self.h, hptr(blob), n, _stream_or_null(stream)))
        return blob[:n]

    def set_queries(self, queries, stream=None):
        codes = np.ascontiguousarray(queries.codes, dtype=np.uint8)
        offs = np.ascontiguousarray(queries.offsets, dtype=np.uint32)
        lens = np.ascontiguousarray(queries.lengths, dtype=np.uint32)
        cut = np.ascontiguousarray(queries.cutoffs, dtype=np.int32)
        trig = np.ascontiguousarray(queries.triggers, dtype=np.int32)
        check(lib().gzb_engine_set_queries(self.h, hptr(codes), len(codes), hptr(offs),
                                           hptr(lens), int(queries.number), hptr(cut),
                                           hptr(trig), _stream_or_null(stream)))
        self.number_queries = int(queries.number)

    def set_protein_queries(self, codes, offsets, lengths, filter=True, ungapped_bits=7.0,
                            trigger_bits=22.0, stream=None):
        """Raw protein queries in the engine layout (codes from
        encode_protein_for_seg) prepared on the device -- SEG when filter,
        per-query cutoffs -- and set (gzb_engine_set_protein_queries).
        Returns the (cutoffs, triggers) host arrays."""
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        offs = np.ascontiguousarray(offsets, dtype=np.uint32)
        lens = np.ascontiguousarray(lengths, dtype=np.uint32)
        n = len(offs)
        cut, trig = np.zeros(n, np.int32), np.zeros(n, np.int32)
        check(lib().gzb_engine_set_protein_queries(
            self.h, hptr(codes), len(codes), hptr(offs), hptr(lens), n, 1 if filter else 0,
            float(ungapped_bits), float(trigger_bits), hptr(cut), hptr(trig),
            _stream_or_null(stream)))
        self.number_queries = n
        return cut, trig

    def set_translated_queries(self, dna, offsets, filter=True, ungapped_bits=7.0,
                               trigger_bits=22.0, stream=None):
        """Reads (ASCII bases back to back, number_reads + 1 offsets)
        translated, SEG-masked (filter) and given their cutoffs on the device
        and set as the query set (gzb_engine_set_translated_queries).
        Returns the (cutoffs, triggers) host arrays."""
        dna = np.ascontiguousarray(dna, dtype=np.uint8)
        offs = np.ascontiguousarray(offsets, dtype=np.uint64)
        n = len(offs) - 1
        cut, trig = np.zeros(n, np.int32), np.zeros(n, np.int32)
        check(lib().gzb_engine_set_translated_queries(
            self.h, hptr(dna), hptr(offs), n, 1 if filter else 0, float(ungapped_bits),
            float(trigger_bits), hptr(cut), hptr(trig), _stream_or_null(stream)))
        self.number_queries = n
        return cut, trig

    def presearch(self, schedule=SCHEDULE_PLAIN, stream=None):
        check(lib().gzb_engine_presearch(self.h, int(schedule), _stream_or_null(stream)))

    def reset_results(self, stream=None):
        check(lib().gzb_engine_reset_results(self.h, _stream_or_null(stream)))

    def result_rows(self, stream=None):
        """The merged lists in the ABI's layout: (counts[number_queries],
        records[number_queries * max_number_results], RESULT_DTYPE)."""
        b = int(self.params[0]["max_number_results"])
        counts = np.zeros(self.number_queries, np.uint32)
        res = np.zeros(self.number_queries * b, RESULT_DTYPE)
        check(lib().gzb_engine_get_results(self.h, hptr(counts), hptr(res),
                                           _stream_or_null(stream)))
        return counts, res

    def results(self, stream=None):
        b = int(self.params[0]["max_number_results"])
        counts, res = self.result_rows(stream)
        res = res.reshape(self.number_queries, b)
        return [res[i, :counts[i]].copy() for i in range(self.number_queries)]

    def build_alignments(self, stream=None):
        """The build results step for the resident chunk: per query its
        results with alignment length, mismatches, gap openings and gap
        extensions (alignment_length 0 for results of other chunks)."""
        b = int(self.params[0]["max_number_results"])
        counts = np.zeros(self.number_queries, np.uint32)
        out = np.zeros(self.number_queries * b, ALIGNMENT_DTYPE)
        check(lib().gzb_engine_build_alignments(self.h, hptr(counts), hptr(out),
                                                _stream_or_null(stream)))
        out = out.reshape(self.number_queries, b)
        return [out[i, :counts[i]].copy() for i in range(self.number_queries)]

    def counters(self):
        c = (C.c_uint64 * 9)()
        check(lib().gzb_engine_get_counters(self.h, C.byref(c)))
        return dict(zip(COUNTER_NAMES, [int(v) for v in c]))

    def stage_ms(self):
        t = (C.c_float * 7)()
        check(lib().gzb_engine_get_stage_ms(self.h, C.byref(t)))
        return dict(zip(("lookup", "seed_ungapped", "chain", "gapped", "merge", "total",
                         "seed_kernels"), [float(v) for v in t]))

    def hits(self, stream=None):
        n = C.c_uint64()
        check(lib().gzb_engine_get_hits(self.h, None, None, None, 0, C.byref(n),
                                        _stream_or_null(stream)))
        k = n.value
        a, b, c = (np.zeros(k, np.uint32) for _ in range(3))
        check(lib().gzb_engine_get_hits(self.h, hptr(a), hptr(b), hptr(c), k, C.byref(n),
                                        _stream_or_null(stream)))
        return a, b, c

    def list_arrays(self, stream=None):
        out = {}
        for i, name in enumerate(LIST_NAMES):
            n = C.c_uint64()
            check(lib().gzb_engine_get_list_array(self.h, i, None, 0, C.byref(n),
                                                  _stream_or_null(stream)))
            a = np.zeros(n.value, np.uint32)
            check(lib().gzb_engine_get_list_array(self.h, i, hptr(a), n.value, C.byref(n),
                                                  _stream_or_null(stream)))
            out[name] = a
        return out

    # ---- cost model of the gapped stage
    def set_logging(self, enable=True, capacity=1 << 24):
        check(lib().gzb_engine_set_logging(self.h, int(bool(enable)), int(capacity)))

    def get_log(self):
        n = C.c_uint64()
        check(lib().gzb_engine_get_log(self.h, None, None, 0, C.byref(n)))
        k = n.value
        x = np.zeros((k, COST_FEATURES), np.float32)
        y = np.zeros(k, np.float32)
        check(lib().gzb_engine_get_log(self.h, hptr(x), hptr(y), k, C.byref(n)))
        return x, y

    def train_cost_model(self, epochs=4, batch=4096, lr=3e-3, seed=0, init=None):
        p = cost_model_init(seed) if init is None else np.array(init, np.float32)
        loss = C.c_float()
        check(lib().gzb_engine_train_cost_model(self.h, int(epochs), int(batch), float(lr),
                                                int(seed), hptr(p), C.byref(loss)))
        return p, float(loss.value)

    def set_cost_model(self, params):
        if params is None:
            check(lib().gzb_engine_set_cost_model(self.h, None))
        else:
            p = np.ascontiguousarray(params, np.float32)
            check(lib().gzb_engine_set_cost_model(self.h, hptr(p)))

    def autotune(self, schedule, candidates=(1, 2, 4, 8, 12, 16, 24), which=TILE_BOOK_THRESHOLD,
                 stream=None):
        """Picks the fastest value of tile parameter `which` for `schedule` on
        the resident workload and keeps it for that schedule; returns (chosen
        value, {candidate: gapped-stage ms}).  Clears the results."""
        cand = np.array(candidates, np.int32)
        ms = np.zeros(len(cand), np.float32)
        best = C.c_int()
        check(lib().gzb_engine_autotune(self.h, int(schedule), int(which), hptr(cand), len(cand),
                                        C.byref(best), hptr(ms), _stream_or_null(stream)))
        return int(best.value), {int(c): float(m) for c, m in zip(cand, ms)}

    def set_tile(self, schedule, which, value):
        """Tile of `schedule` (-1: the process-wide default)."""
        check(lib().gzb_engine_set_tile(self.h, int(schedule), int(which), int(value)))

    def tile(self, schedule, which):
        v = C.c_int()
        check(lib().gzb_engine_get_tile(self.h, int(schedule), int(which), C.byref(v)))
        return int(v.value)

    def extension_costs(self, predicted=True):
        """(predicted log2(1+cells) or None, true DP cells) of the last
        work-queue run, in extension order."""
        n = C.c_uint64()
        check(lib().gzb_engine_get_extension_costs(self.h, None, None, 0, C.byref(n), None))
        cells = np.zeros(n.value, np.uint32)
        pred = np.zeros(n.value, np.float32) if predicted else None
        check(lib().gzb_engine_get_extension_costs(
            self.h, hptr(pred) if predicted else None, hptr(cells), n.value, C.byref(n), None))
        return pred, cells

    def schedule_stats(self):
        err = C.c_float()
        n = C.c_uint64()
        check(lib().gzb_engine_get_schedule_stats(self.h, C.byref(err), C.byref(n)))
        return float(err.value), int(n.value)

    def index_arrays(self, stream=None):
        out = {}
        for i, name in enumerate(INDEX_NAMES):
            n = C.c_uint64()
            check(lib().gzb_engine_get_index_array(self.h, i, None, 0, C.byref(n),
                                                   _stream_or_null(stream)))
            a = np.zeros(n.value, np.uint32)
            check(lib().gzb_engine_get_index_array(self.h, i, hptr(a), n.value, C.byref(n),
                                                   _stream_or_null(stream)))
            out[name] = a
        return out


def _stream_or_null(stream):
    if stream is None:
        return None
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


# -- query preparation: six-frame translation ---------------------------------
def merge_chunk_results(params, chunk_counts, chunk_records, counts, records):
    """gzb_merge_chunk_results: one chunk's lists (counts, RESULT_DTYPE rows
    of max_number_results) merged in place into the running lists."""
    rec = np.array([params], dtype=params.dtype)
    b = int(params["max_number_results"])
    nq = len(counts)
    for a, dt, n in ((chunk_counts, np.uint32, nq), (counts, np.uint32, nq),
                     (chunk_records, RESULT_DTYPE, nq * b), (records, RESULT_DTYPE, nq * b)):
        assert a.dtype == dt and a.flags.c_contiguous and len(a) == n
    check(lib().gzb_merge_chunk_results(C.c_void_p(rec.ctypes.data), nq, hptr(chunk_counts),
                                        hptr(chunk_records), hptr(counts), hptr(records)))


def params_from_reference_common(scp, params):
    """A copy of `params` with the seed-index fields the reference's .scp
    file (its bytes) stores; host only."""
    rec = np.array([params], dtype=params.dtype)
    scp = np.ascontiguousarray(np.frombuffer(scp, np.uint8) if isinstance(scp, bytes) else scp,
                               dtype=np.uint8)
    check(lib().gzb_params_from_reference_common(hptr(scp), scp.nbytes,
                                                 C.c_void_p(rec.ctypes.data)))
    return rec[0]


def index_blob_from_reference(params, sdp, db):
    """The reference's on-disk seed-searcher index of chunk `db` (the bytes
    of its .sdp file) as an index blob for PresearchEngine.set_database(db,
    index=...).  Host only: no device is needed."""
    rec = np.array([params], dtype=params.dtype)
    sdp = np.ascontiguousarray(np.frombuffer(sdp, np.uint8) if isinstance(sdp, bytes) else sdp,
                               dtype=np.uint8)
    codes = np.ascontiguousarray(db.codes, dtype=np.uint8)
    offs = np.ascontiguousarray(db.offsets, dtype=np.uint32)
    n = C.c_uint64()
    args = (C.c_void_p(rec.ctypes.data), hptr(sdp), sdp.nbytes, hptr(codes), len(codes),
            hptr(offs), int(db.number_sequences))
    check(lib().gzb_index_blob_from_reference(*args, None, 0, C.byref(n)))
    blob = np.zeros(int(n.value), np.uint8)
    check(lib().gzb_index_blob_from_reference(*args, hptr(blob), blob.nbytes, C.byref(n)))
    return blob


def translated_query_length(length):
    """Codes of a read's translated query, both delimiters included
    (TranslatedDnaQuery::GetSequenceLength, src/translated_dna_query.h:24-31;
    2 for a read shorter than 3 bases)."""
    return int(lib().gzb_translated_query_length(int(length)))


def translated_layout(lengths):
    """Shared-delimiter layout of the translated queries of reads with these
    lengths: (out_offsets uint64, query lengths uint32, total codes)."""
    n = np.asarray(lengths, dtype=np.int64)
    ql = np.where(n < 3, 2, 7 + 6 * (n // 3)).astype(np.int64)
    offs = np.zeros(len(ql), dtype=np.uint64)
    if len(ql) > 1:
        offs[1:] = np.cumsum(ql - 1)[:-1]
    total = int((ql - 1).sum()) + 1 if len(ql) else 0
    return offs, ql.astype(np.uint32), total


def translate_dna_queries_async(d_dna, d_offsets, d_lengths, number_reads, d_out_offsets,
                                d_out, delimiter, stream=None):
    """gzb_translate_dna_queries on device buffers (addresses or tensors)."""
    check(lib().gzb_translate_dna_queries(dptr(d_dna), dptr(d_offsets), dptr(d_lengths),
                                          int(number_reads), dptr(d_out_offsets),
                                          int(delimiter), dptr(d_out),
                                          stream_handle(stream)))


def translate_reads(dna, offsets, delimiter, device="cuda", stream=None):
    """Translates reads on the GPU.  dna: uint8 ASCII bases of all reads
    back to back; offsets: number_reads + 1 read boundaries.  Returns the
    translated queries in the engine's shared-delimiter layout as host
    arrays (codes uint8, offsets uint32, lengths uint32)."""
    import torch
    offsets = np.asarray(offsets, dtype=np.uint64)
    n = len(offsets) - 1
    lengths = np.diff(offsets).astype(np.uint32)
    out_offs, qlen, total = translated_layout(lengths)
    if n == 0:
        return np.zeros(0, np.uint8), np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    d_dna = torch.from_numpy(np.require(dna, np.uint8, ["C", "W"])).to(device)
    d_offs = torch.from_numpy(offsets[:-1].view(np.int64).copy()).to(device)
    d_lens = torch.from_numpy(lengths.view(np.int32).copy()).to(device)
    d_out_offs = torch.from_numpy(out_offs.view(np.int64).copy()).to(device)
    d_out = torch.empty(total, dtype=torch.uint8, device=device)
    translate_dna_queries_async(d_dna, d_offs, d_lens, n, d_out_offs, d_out, delimiter,
                                stream)
    codes = d_out.cpu().numpy()
    return codes, out_offs.astype(np.uint32), qlen


# -- query preparation: per-query Karlin cutoffs ---------------------------------
def query_karlin_cutoffs_async(d_codes, d_offsets, d_lengths, number_queries, matrix,
                               d_cutoffs, d_triggers, d_karlin=None, ungapped_bits=7.0,
                               trigger_bits=22.0, stream=None):
    """gzb_query_karlin_cutoffs on device buffers; matrix is a host
    (n, n) int32 score matrix."""
    m = np.ascontiguousarray(matrix, dtype=np.int32)
    check(lib().gzb_query_karlin_cutoffs(dptr(d_codes), dptr(d_offsets), dptr(d_lengths),
                                         int(number_queries), hptr(m), int(m.shape[0]),
                                         float(ungapped_bits), float(trigger_bits),
                                         dptr(d_cutoffs), dptr(d_triggers), dptr(d_karlin),
                                         stream_handle(stream)))


def query_karlin_cutoffs(codes, offsets, lengths, matrix=None, ungapped_bits=7.0,
                         trigger_bits=22.0, device="cuda"):
    """Per-query ungapped X-drop and gapped-extension trigger computed on
    the GPU for queries laid out in host arrays (whole queries, delimiters
    included).  Returns (cutoffs int32, triggers int32, karlin float32 (n, 3)
    = lambda, K, H)."""
    import torch
    from . import params as P
    m = P.blosum62() if matrix is None else matrix
    n = len(offsets)
    if n == 0:
        return np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, 3), np.float32)
    d_codes = torch.from_numpy(np.ascontiguousarray(codes, dtype=np.uint8)).to(device)
    d_offs = torch.from_numpy(np.asarray(offsets, dtype=np.int64).copy()).to(device)
    d_lens = torch.from_numpy(np.asarray(lengths, dtype=np.uint32).view(np.int32).copy()).to(device)
    d_cut = torch.empty(n, dtype=torch.int32, device=device)
    d_trig = torch.empty(n, dtype=torch.int32, device=device)
    d_k = torch.empty(3 * n, dtype=torch.float32, device=device)
    query_karlin_cutoffs_async(d_codes, d_offs, d_lens, n, m, d_cut, d_trig, d_k,
                               ungapped_bits, trigger_bits)
    return d_cut.cpu().numpy(), d_trig.cpu().numpy(), d_k.cpu().numpy().reshape(n, 3)


# -- query preparation: SEG and whole-query preparation --------------------------
SEG_WINDOW = 12


def seg_translated_queries_async(d_queries, d_query_offsets, d_read_lengths, number_queries,
                                 d_status=None, stream=None):
    check(lib().gzb_seg_translated_queries(dptr(d_queries), dptr(d_query_offsets),
                                           dptr(d_read_lengths), int(number_queries),
                                           dptr(d_status), stream_handle(stream)))


def seg_protein_queries_async(d_codes, d_offsets, d_lengths, number_queries, d_status=None,
                              stream=None):
    check(lib().gzb_seg_protein_queries(dptr(d_codes), dptr(d_offsets), dptr(d_lengths),
                                        int(number_queries), dptr(d_status),
                                        stream_handle(stream)))


def encode_protein_for_seg(letters):
    """Protein letters -> codes for gzb_seg_protein_queries: lower-case
    letters (which the reference's SEG does not count) get code + 32."""
    from . import params as P
    raw = np.frombuffer(bytes(letters), dtype=np.uint8)
    codes = P.encode(bytes(raw).decode("latin-1").upper()).astype(np.uint8)
    lower = (raw >= ord("a")) & (raw <= ord("z"))
    codes[lower] += 32
    return codes


def prepare_translated_queries(dna, offsets, filter=True, matrix=None, ungapped_bits=7.0,
                               trigger_bits=22.0, device="cuda"):
    """Query preparation of translated-DNA searches on the GPU: six-frame
    translation, SEG (filter=True, the aln default) and per-query cutoffs.
    dna: uint8 ASCII bases back to back; offsets: number_reads + 1 read
    boundaries.  Returns host arrays (codes, offsets uint32, lengths uint32,
    cutoffs int32, triggers int32) in the engine's query layout."""
    import torch
    from . import params as P
    offsets = np.asarray(offsets, dtype=np.uint64)
    n = len(offsets) - 1
    lengths = np.diff(offsets).astype(np.uint32)
    out_offs, qlen, total = translated_layout(lengths)
    if n == 0:
        z = np.zeros(0, np.uint32)
        return np.zeros(0, np.uint8), z, z, z.astype(np.int32), z.astype(np.int32)
    d_dna = torch.from_numpy(np.require(dna, np.uint8, ["C", "W"])).to(device)
    d_offs = torch.from_numpy(offsets[:-1].view(np.int64).copy()).to(device)
    d_lens = torch.from_numpy(lengths.view(np.int32).copy()).to(device)
    d_qoffs = torch.from_numpy(out_offs.view(np.int64).copy()).to(device)
    d_qlen = torch.from_numpy(qlen.view(np.int32).copy()).to(device)
    d_out = torch.empty(total, dtype=torch.uint8, device=device)
    d_status = torch.zeros(1, dtype=torch.int32, device=device)
    d_cut = torch.empty(n, dtype=torch.int32, device=device)
    d_trig = torch.empty(n, dtype=torch.int32, device=device)
    translate_dna_queries_async(d_dna, d_offs, d_lens, n, d_qoffs, d_out, P.DELIMITER)
    if filter:
        seg_translated_queries_async(d_out, d_qoffs, d_lens, n, d_status)
    m = P.blosum62() if matrix is None else matrix
    query_karlin_cutoffs_async(d_out, d_qoffs, d_qlen, n, m, d_cut, d_trig, None,
                               ungapped_bits, trigger_bits)
    if int(d_status.item()) != 0:
        raise GzbError(f"SEG left {int(d_status.item())} frames unmasked")
    return (d_out.cpu().numpy(), out_offs.astype(np.uint32), qlen, d_cut.cpu().numpy(),
            d_trig.cpu().numpy())


def prepare_protein_queries(codes, offsets, lengths, filter=True, matrix=None,
                            ungapped_bits=7.0, trigger_bits=22.0, device="cuda"):
    """Query preparation of protein searches on the GPU: SEG (filter=True,
    the aln default) and per-query cutoffs, for queries in the engine layout
    (codes from encode_protein_for_seg keep lower-case letters out of SEG's
    compositions).  Returns host arrays (codes, cutoffs, triggers)."""
    import torch
    from . import params as P
    offsets = np.asarray(offsets, dtype=np.uint64)
    lengths = np.asarray(lengths, dtype=np.uint32)
    n = len(offsets)
    if n == 0:
        return np.zeros(0, np.uint8), np.zeros(0, np.int32), np.zeros(0, np.int32)
    d_codes = torch.from_numpy(np.ascontiguousarray(codes, dtype=np.uint8)).to(device)
    d_offs = torch.from_numpy(offsets.view(np.int64).copy()).to(device)
    d_lens = torch.from_numpy(lengths.view(np.int32).copy()).to(device)
    d_status = torch.zeros(1, dtype=torch.int32, device=device)
    d_cut = torch.empty(n, dtype=torch.int32, device=device)
    d_trig = torch.empty(n, dtype=torch.int32, device=device)
    m = P.blosum62() if matrix is None else matrix
    if filter:
        seg_protein_queries_async(d_codes, d_offs, d_lens, n, d_status)
    query_karlin_cutoffs_async(d_codes, d_offs, d_lens, n, m, d_cut, d_trig, None,
                               ungapped_bits, trigger_bits)
    cut, trig = d_cut.cpu().numpy(), d_trig.cpu().numpy()
    if filter:
        # a protein the filter refuses (shorter than the window) is held as
        # [delimiter] + zeros, its last code 0 rather than a delimiter, and
        # its statistics are those of that buffer
        short = np.flatnonzero(lengths - 2 < SEG_WINDOW)
        if len(short):
            bufs = [np.concatenate([[P.DELIMITER], np.zeros(int(lengths[i]) - 1, np.uint8)])
                    for i in short]
            sc, so, sl = (np.concatenate(bufs).astype(np.uint8),
                          np.concatenate([[0], np.cumsum([len(b) for b in bufs])[:-1]]),
                          np.array([len(b) for b in bufs], np.uint32))
            c2, t2, _ = query_karlin_cutoffs(sc, so, sl, m, ungapped_bits, trigger_bits,
                                             device)
            cut[short], trig[short] = c2, t2
    if int(d_status.item()) != 0:
        raise GzbError(f"SEG left {int(d_status.item())} queries unmasked")
    return d_codes.cpu().numpy(), cut, trig


# -- the final hit table --------------------------------------------------------------
def gapped_karlin_parameters(matrix_name="BLOSUM62", gap_open=11, gap_extension=1):
    """(lambda, K, H, alpha, beta) of the gapped protein search."""
    lam, k, h = C.c_float(), C.c_float(), C.c_float()
    alpha, beta = C.c_double(), C.c_double()
    check(lib().gzb_gapped_karlin_parameters(matrix_name.encode(), int(gap_open),
                                             int(gap_extension), C.byref(lam), C.byref(k),
                                             C.byref(h), C.byref(alpha), C.byref(beta)))
    return lam.value, k.value, h.value, alpha.value, beta.value


def search_space(query_length, db_length, db_sequences, karlin):
    lam, k, _, alpha, beta = karlin
    return int(lib().gzb_search_space(int(query_length), int(db_length), int(db_sequences),
                                      lam, k, alpha, beta))


def evalue(score, space, karlin):
    return float(lib().gzb_evalue(int(score), int(space), karlin[0], karlin[1]))


def bit_score(score, karlin):
    return float(lib().gzb_bit_score(int(score), karlin[0], karlin[1]))


def _rows(results):
    nq = len(results)
    stride = max([len(r) for r in results] + [1])
    counts = np.array([len(r) for r in results], np.uint32)
    rows = np.zeros(nq * stride, ALIGNMENT_DTYPE)
    for i, r in enumerate(results):
        rows[i * stride:i * stride + len(r)] = r
    return stride, counts, rows


def sort_alignments(results, db_offsets, number_subjects, dna_lengths=None):
    """Each query's alignment records (build_alignments() rows in merged
    order) in the order the reference writes them (gzb_sort_alignments:
    AlignerCommon::ResultGreaterScore over the printed coordinates)."""
    nq = len(results)
    if nq == 0:
        return []
    stride, counts, rows = _rows(results)
    offs = np.ascontiguousarray(db_offsets, dtype=np.uint32)
    dna = None if dna_lengths is None else np.ascontiguousarray(dna_lengths, dtype=np.uint32)
    check(lib().gzb_sort_alignments(nq, stride, hptr(counts), hptr(rows), int(number_subjects),
                                    hptr(offs), hptr(dna)))
    rows = rows.reshape(nq, stride)
    return [rows[i, :counts[i]].copy() for i in range(nq)]


def hit_table(results, query_names, subject_names, db_offsets, db_length, db_sequences,
              query_real_lengths, dna_lengths=None, karlin=None):
    """The `aln` tabular output (AlignerCommon::WriteOutput,
    src/aligner_common.h:344-394) of build_alignments() results, written by
    the library (gzb_write_hit_table): per result query name, subject name,
    identity %, alignment length, mismatches, gap openings, query start and
    end (bases of the read for translated queries), subject start and end,
    E-value and normalized score, tab separated, numbers as C++ streams
    print them; returns the lines.  db_offsets: the chunk's first-residue
    offsets; db_length / db_sequences: residues and sequences of the whole
    database; query_real_lengths: residues (a read's bases / 3 for a
    translated query); dna_lengths: the reads' bases for translated queries
    (None for protein queries)."""
    if karlin is None:
        karlin = gapped_karlin_parameters()
    lam, k, _, alpha, beta = karlin
    nq = len(results)
    stride = max([len(r) for r in results] + [1])
    counts = np.array([len(r) for r in results], np.uint32)
    rows = np.zeros(nq * stride, ALIGNMENT_DTYPE)
    for i, r in enumerate(results):
        rows[i * stride:i * stride + len(r)] = r
    qn = (C.c_char_p * max(nq, 1))(*[n.encode() for n in query_names[:nq]])
    sn = (C.c_char_p * max(len(subject_names), 1))(*[n.encode() for n in subject_names])
    offs = np.ascontiguousarray(db_offsets, dtype=np.uint32)
    real = np.ascontiguousarray(query_real_lengths, dtype=np.uint32)
    dna = None if dna_lengths is None else np.ascontiguousarray(dna_lengths, dtype=np.uint32)
    args = [nq, stride, hptr(counts), hptr(rows), qn, sn, len(subject_names), hptr(offs),
            int(db_length), int(db_sequences), hptr(real), hptr(dna), lam, k, alpha, beta]
    n = C.c_uint64()
    check(lib().gzb_write_hit_table(*args, None, 0, C.byref(n)))
    out = C.create_string_buffer(max(int(n.value), 1))
    check(lib().gzb_write_hit_table(*args, out, n.value, C.byref(n)))
    return out.raw[:n.value].decode().splitlines()
