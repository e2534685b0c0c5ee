"""The multi-rank host logic of bench.py on CPU, two `gloo` ranks: each rank
draws its own shard (weak scaling, no data-path collective), the job's time
is the max over ranks, and the whole-job value counts every rank's
matrices.  No GPU: the ranks only exchange one float."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    from datetime import timedelta
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ns, seed = bench.shard(rank, 2000)
        # A rank's "step time": rank 1 is the slow one.
        t = 0.25 + 0.5 * rank
        slowest = bench.max_over_ranks(t, world, torch.device("cpu"))
        dist.barrier()
        out.put((rank, slowest, int(ns.sum()), int(ns.min()), int(ns.max()), seed))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, ROOT)
    import bench
    (r0, m0, s0, lo0, hi0, seed0), (r1, m1, s1, lo1, hi1, seed1) = res
    assert m0 == m1 == 0.75            # both ranks see the slowest rank's time
    assert s0 != s1 and seed0 != seed1  # two different shards
    assert bench.NMIN <= min(lo0, lo1) and max(hi0, hi1) <= bench.NMAX
    # The whole-job value bench.py reports: both ranks' shards over the
    # slowest rank's time.
    assert bench.job_value(2, 2000, 3, m0) == pytest.approx(16000.0)
    assert bench.job_value(1, 2000, 3, 0.25) == pytest.approx(24000.0)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(1.5, 1, None) == 1.5
    ns, seed = bench.shard(0, 100)
    assert len(ns) == 100 and seed == bench.SEED
    np.testing.assert_array_equal(ns, bench.draw_sizes(100, bench.SEED))
