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
        ns, seed = bench.shard(rank, 2000, world)
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


def test_partitioner_balances_cost_and_covers_every_matrix():
    """nmx_batched_partition (host only): every matrix on exactly one device,
    per-device predicted cost within 0.1 % of the mean for a 100k-matrix
    batch over 8 devices, deterministic, and the split bench.py's ranks take
    is a partition of the job's sizes."""
    sys.path.insert(0, ROOT)
    from numax_b200 import build
    build.build()
    from numax_b200.batched import partition
    import bench
    rng = np.random.Generator(np.random.PCG64(8))
    ns = rng.integers(8, 129, size=100_000).astype(np.int32)
    for ndev in (1, 2, 3, 8):
        dev_of, cost = partition(ns, ndev, 4)
        assert dev_of.min() >= 0 and dev_of.max() < ndev
        assert np.bincount(dev_of, minlength=ndev).sum() == len(ns)
        assert cost.max() / cost.mean() <= 1.001, cost
        n64 = ns.astype(np.float64)
        c = n64 ** 3 / 3 + 8 * n64 ** 2 + 96 * n64 ** 2
        np.testing.assert_allclose(cost, np.bincount(dev_of, weights=c, minlength=ndev))
        again, _ = partition(ns, ndev, 4)
        np.testing.assert_array_equal(dev_of, again)
    # bench.py's shards: disjoint, together the whole job's size draw.
    world = 4
    parts = [bench.shard(r, 1000, world)[0] for r in range(world)]
    np.testing.assert_array_equal(np.sort(np.concatenate(parts)),
                                  np.sort(bench.draw_sizes(4000, bench.SEED)))
    # Rejects bad arguments without a device.
    from numax_b200 import _lib
    with pytest.raises(_lib.NmxError):
        partition(np.array([0], dtype=np.int32), 2)
    with pytest.raises(_lib.NmxError):
        partition(ns[:10], 0)
