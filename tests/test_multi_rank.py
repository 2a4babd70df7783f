"""Multi-rank plumbing of the benchmark on CPU ranks (gloo, world size 2):
the max-over-ranks timing, the ray totals, and the split of a scene batch
across ranks.  The path itself has no collective: ranks are replicas (or own
disjoint scenes) and only the timing is exchanged."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import rayengine_b200 as rb

    dist = bench.init_dist(world, "gloo")
    r, w, _ = bench.dist_env()
    slowest = bench.max_over_ranks(1.5 * (r + 1), w, device="cpu")
    total = bench.sum_over_ranks(100 * (r + 1), w, device="cpu")
    specs = rb.configs.BatchConfig().specs()
    mine = rb.configs.BatchConfig.shard(specs, r, w)
    bench.barrier(w)
    q.put((r, slowest, total, [(s["seed"], s["width"] * s["height"]) for s in mine]))
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
    assert [o[1] for o in out] == [3.0, 3.0]  # both see the slowest rank's time
    assert [o[2] for o in out] == [300, 300]
    a, b = out[0][3], out[1][3]
    seeds = [s for s, _ in a] + [s for s, _ in b]
    assert len(seeds) == len(set(seeds)) == 32  # disjoint, complete
    pa, pb = sum(p for _, p in a), sum(p for _, p in b)
    assert abs(pa - pb) <= 1920 * 1080  # balanced to within one largest scene


def test_single_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench
    import rayengine_b200 as rb

    assert bench.max_over_ranks(2.5, 1) == 2.5
    assert bench.sum_over_ranks(7, 1) == 7
    specs = rb.configs.BatchConfig().specs()
    assert rb.configs.BatchConfig.shard(specs, 0, 1) == specs
