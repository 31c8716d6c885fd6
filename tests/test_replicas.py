"""The multi-GPU path of the benchmark on the CPU: two gloo ranks (the same
code the nccl ranks run) meet at the barrier, agree on the slowest rank's
times and report the whole-job rate."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from gzb.replicas import Replicas
    r = Replicas("gloo", timeout_s=60)
    r.barrier()
    # rank 0 is the slow one for the first figure, rank 1 for the second
    m = r.max([100.0 - 10 * rank, 50.0 + 5 * rank])
    rate = r.throughput(1000, 3, m[0])
    r.barrier()
    r.close()
    out.put((rank, m, rate))


def test_two_gloo_ranks_agree_on_the_slowest_time():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, rate in got:
        assert m == [100.0, 55.0], (rank, m)
        assert rate == pytest.approx(2 * 1000 * 3 / 0.1)


def test_single_process_is_local():
    from gzb.replicas import Replicas
    env = {k: os.environ.pop(k, None) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    try:
        r = Replicas("gloo")
        assert r.world == 1 and r.dist is None
        assert r.max([1.0, 2.0]) == [1.0, 2.0]
        assert r.throughput(10, 2, 1000.0) == 20.0
        r.close()
    finally:
        for k, v in env.items():
            if v is not None:
                os.environ[k] = v
