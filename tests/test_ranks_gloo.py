"""The benchmark's multi-rank logic on CPU: two gloo ranks, each with its own
seeded domain and device time; the max over ranks and the weak-scaling value
agree on both ranks."""
import os

import pytest


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from roundabout_b200.ranks import max_over_ranks, rank_seed, weak_scaling_value
    from roundabout_b200.synthetic import make_columns

    cols = make_columns(16, 12, 8, ntracers=2, seed=rank_seed(1234, rank), land_frac=0.3)
    my_ms = 10.0 + 5.0 * rank
    ms = max_over_ranks(my_ms, dist, device="cpu")
    value = weak_scaling_value(16 * 12 * 8, 3, world, ms)
    q.put((rank, ms, value, float(cols.tracers[1].sum())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    import socket

    import torch.multiprocessing as mp

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ms0, v0, s0), (r1, ms1, v1, s1) = out
    assert ms0 == ms1 == 15.0                      # the slowest rank's time on both
    assert v0 == v1 == pytest.approx(16 * 12 * 8 * 3 * 2 / 0.015)
    assert s0 != s1                                # independently seeded domains
