"""bench.py's multi-rank plumbing on CPU with two gloo ranks: timings combine as the
max over ranks, every rank reaches the barrier, each rank gets its own piece seed, and
the reference arm does no work on ranks other than 0."""
import multiprocessing as mp
import os
import socket

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        slowest = bench.max_over_ranks(100.0 + 7 * rank, world)
        bench.barrier(world)
        r, w, local = bench.dist_env()

        class Args:
            gpus, steps, warmup, seed = world, 1, 0, 0
        ref = bench.run_reference(Args) if rank != 0 else None  # rank 0 would run the CPU leg
        q.put((rank, slowest, r, w, local, bench.rank_seed(5, rank), ref))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [107.0, 107.0]          # max over ranks, on every rank
    assert [(o[2], o[3], o[4]) for o in out] == [(0, 2, 0), (1, 2, 1)]
    assert [o[5] for o in out] == [5, 6]                   # a piece of its own per rank
    assert out[1][6] is None                               # reference arm: rank 1 does nothing
