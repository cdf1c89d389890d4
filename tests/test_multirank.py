"""bench.py's multi-rank plumbing on CPU with two gloo ranks: timings combine as the
max over ranks, every rank reaches the barrier, each rank gets its own piece seed, the
reference arm does no work on ranks other than 0, and one batch splits across the ranks
(longest first by unknowns: every piece on exactly one rank, loads within the LPT bound)
with its statistics summed on every rank."""
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

    import numpy as np

    sys.path[:0] = [ROOT, os.path.join(ROOT, "parallax-world_b200")]
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
        # one batch split across the ranks: the same split on every rank
        from statics_cuda import shard
        weights = [int(v) for v in np.random.default_rng(3).integers(1000, 50000, size=101)]
        split = shard.lpt_split(weights, world)
        # this rank's solves (made up), their statistics summed over the ranks
        infos = [{"status": 0, "residual": 1e-9 * (rank + 1), "refinements": rank, "iterations": 40 + rank}
                 for _ in split[rank]]
        infos[0]["status"] = 1 if rank == 1 else 0
        stats = bench.batch_stats(infos, 1e-8, world)
        q.put((rank, slowest, r, w, local, bench.rank_seed(5, rank), ref, split, weights, stats))
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
    split, weights = out[0][7], out[0][8]
    assert out[1][7] == split                              # every rank computes the same split
    assert sorted(i for s in split for i in s) == list(range(len(weights)))
    loads = [sum(weights[i] for i in s) for s in split]
    assert max(loads) <= sum(weights) / 2 + max(weights)   # LPT: mean load plus the heaviest piece
    assert max(loads) - min(loads) <= max(weights)
    for o in out:                                          # statistics summed / maxed over ranks
        st = o[9]
        assert st["pieces"] == len(weights)
        assert st["failed"] == 1
        assert st["replaced"] == len(split[1])
        assert st["max_true_residual"] == 2e-9
