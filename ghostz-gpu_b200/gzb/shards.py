"""Database chunks spread over GPUs, one process per GPU.

The path's one exchange step: the reference's chunk loop
(src/aligner_gpu_presearch_thread.cpp:214-640) merges every chunk's results
into the per-query top-b lists with AlignerCommon::AddResults
(src/aligner_common.h:147-274).  Here rank r searches chunks r, r + N,
r + 2N, ... with its results reset before each chunk, the per-chunk lists
are all-gathered (NCCL between GPUs, gloo between CPU processes), every
rank merges its slice of the queries in chunk order with
gzb_merge_chunk_results, which gives exactly the lists of one engine
searching every chunk in turn, and the merged slices are all-gathered.
"""
import numpy as np

from . import native as N

RECORD_WORDS = N.RESULT_DTYPE.itemsize // 4


def chunks_of(rank, world, n_chunks):
    """The chunks rank `rank` of `world` searches."""
    return list(range(rank, n_chunks, world))


def query_range(rank, world, n_queries):
    """The queries [begin, end) rank `rank` of `world` searches when the
    query set is split over GPUs (every query is independent of the others,
    so the split needs no exchange): contiguous, sizes differing by at most
    one."""
    return rank * n_queries // world, (rank + 1) * n_queries // world


def slice_queries(queries, begin, end):
    """Queries begin .. end - 1 of a query set in the engine layout
    (concatenated, shared delimiters) as a query set of their own."""
    from . import workload as W
    if end <= begin:
        return W.Queries(codes=np.full(1, queries.codes[0], np.uint8),
                         offsets=np.zeros(0, np.uint32), lengths=np.zeros(0, np.uint32),
                         cutoffs=np.zeros(0, np.int32), triggers=np.zeros(0, np.int32),
                         sources=np.zeros(0, np.int64))
    o0 = int(queries.offsets[begin])
    o1 = int(queries.offsets[end - 1]) + int(queries.lengths[end - 1])
    src = queries.sources[begin:end] if queries.sources is not None else None
    return W.Queries(codes=np.ascontiguousarray(queries.codes[o0:o1]),
                     offsets=(queries.offsets[begin:end].astype(np.int64) - o0).astype(np.uint32),
                     lengths=np.ascontiguousarray(queries.lengths[begin:end]),
                     cutoffs=np.ascontiguousarray(queries.cutoffs[begin:end]),
                     triggers=np.ascontiguousarray(queries.triggers[begin:end]),
                     sources=src)


def merge_in_order(params, lists, q0=0, q1=None):
    """lists[c] = (counts, records) of chunk c alone; returns the running
    merge of all of them in chunk order, for queries q0 .. q1 - 1."""
    b = int(params["max_number_results"])
    q1 = len(lists[0][0]) if q1 is None else q1
    counts = np.zeros(q1 - q0, np.uint32)
    records = np.zeros((q1 - q0) * b, N.RESULT_DTYPE)
    for chunk_counts, chunk_records in lists:
        N.merge_chunk_results(params, np.ascontiguousarray(chunk_counts[q0:q1]),
                              np.ascontiguousarray(chunk_records[q0 * b:q1 * b]), counts,
                              records)
    return counts, records


class ChunkShards:
    """Rank and world of an initialised torch.distributed process group (or
    one local process when `dist` is None); `device` is where the gathered
    buffers live ("cuda" for NCCL, "cpu" for gloo)."""

    def __init__(self, dist=None, device="cpu"):
        self.dist = dist
        self.device = device
        self.world = dist.get_world_size() if dist is not None else 1
        self.rank = dist.get_rank() if dist is not None else 0

    def exchange(self, params, n_chunks, number_queries, local):
        """local = {chunk id: (counts, records)} for this rank's chunks;
        returns every chunk's lists, indexed by chunk id, on every rank.  All
        ranks take part with equal-sized buffers (chunks a rank does not have
        travel as zeros and are ignored)."""
        b = int(params["max_number_results"])
        nq = int(number_queries)
        words = nq + nq * b * RECORD_WORDS
        per_rank = -(-n_chunks // self.world)
        buf = np.zeros((per_rank, words), np.int32)
        for i, c in enumerate(chunks_of(self.rank, self.world, n_chunks)):
            counts, records = local[c]
            buf[i, :nq] = counts.view(np.int32)
            buf[i, nq:] = np.ascontiguousarray(records, N.RESULT_DTYPE).view(np.int32)
        if self.dist is None:
            gathered = [buf]
        else:
            import torch
            t = torch.from_numpy(buf).to(self.device)
            outs = [torch.empty_like(t) for _ in range(self.world)]
            self.dist.all_gather(outs, t)
            gathered = [o.cpu().numpy() for o in outs]
        lists = [None] * n_chunks
        for r in range(self.world):
            for i, c in enumerate(chunks_of(r, self.world, n_chunks)):
                row = gathered[r][i]
                lists[c] = (row[:nq].view(np.uint32).copy(),
                            row[nq:].copy().view(N.RESULT_DTYPE))
        return lists

    def merged(self, params, lists):
        """The merge of every chunk's lists in chunk order, on every rank:
        each rank merges its own slice of the queries, and the merged slices
        are all-gathered."""
        if self.dist is None:
            return merge_in_order(params, lists)
        import torch
        b = int(params["max_number_results"])
        nq = len(lists[0][0])
        per = -(-nq // self.world)
        q0 = min(self.rank * per, nq)
        q1 = min(q0 + per, nq)
        counts, records = merge_in_order(params, lists, q0, q1)
        buf = np.zeros(per + per * b * RECORD_WORDS, np.int32)
        buf[:q1 - q0] = counts.view(np.int32)
        buf[per:per + (q1 - q0) * b * RECORD_WORDS] = records.view(np.int32)
        t = torch.from_numpy(buf).to(self.device)
        outs = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(outs, t)
        all_counts = np.zeros(nq, np.uint32)
        all_records = np.zeros(nq * b, N.RESULT_DTYPE)
        for r, o in enumerate(outs):
            a0 = min(r * per, nq)
            a1 = min(a0 + per, nq)
            row = o.cpu().numpy()
            all_counts[a0:a1] = row[:a1 - a0].view(np.uint32)
            all_records[a0 * b:a1 * b] = \
                row[per:per + (a1 - a0) * b * RECORD_WORDS].copy().view(N.RESULT_DTYPE)
        return all_counts, all_records

    def search(self, engine, params, chunks, schedule=N.SCHEDULE_BATCHED):
        """Presearch of the engine's resident queries against this rank's
        chunks (each set in turn, results reset before each), then the
        exchange and the merge: (counts, records) of all chunks, on every
        rank."""
        local = {}
        for c in chunks_of(self.rank, self.world, len(chunks)):
            engine.set_database(chunks[c], chunk_id=c)
            engine.reset_results()
            engine.presearch(schedule)
            local[c] = engine.result_rows()
        lists = self.exchange(params, len(chunks), engine.number_queries, local)
        return self.merged(params, lists)
