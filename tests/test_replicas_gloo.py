"""The N>1 replica path of bench.py on CPU: two gloo ranks."""
import os
import socket

import torch.multiprocessing as mp

from scaph_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    srcs = list(range(100, 164))
    mine = replicas.rank_sources(srcs, rank, 10)
    ms = replicas.max_over_ranks(10.0 + rank, world)  # rank 1 is slower
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, mine, ms))


def test_two_gloo_ranks_take_the_slowest_time_and_distinct_sources():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, s0, m0), (_, s1, m1) = res
    assert m0 == m1 == 11.0
    assert s0 != s1 and len(s0) == len(s1) == 10
    assert replicas.aggregate_gteps(world, 10, 1_000_000, 11.0) == 2 * 10 * 1e6 / 0.011 / 1e9


def test_single_rank_identity():
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.rank_sources([1, 2, 3], 0, 5) == [1, 2, 3, 1, 2]
