"""The N > 1 path of bench.py on CPU: world size 2 over gloo.

bench.py --gpus N runs N independent replicas (the single-matrix SVD has no
shard boundary); the whole-job value is all ranks' matrices over the slowest
rank's time (max over ranks).  Here two gloo ranks report different local
times and both must get the same aggregate.
"""

import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    local_ms = [400.0, 1000.0][rank]
    value, tmax = bench.replica_throughput(local_ms, steps=5, world=world, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, value, tmax))


def test_replicas_aggregate_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    got = sorted(q.get(timeout=10) for _ in range(2))
    for p in ps:
        assert p.exitcode == 0
    for _, value, tmax in got:
        assert tmax == 1000.0                      # the slowest rank
        assert value == pytest.approx(2 * 5 / 1.0)  # 10 matrices in 1 s


def test_single_rank_is_local():
    sys.path.insert(0, ROOT)
    import bench
    v, t = bench.replica_throughput(250.0, steps=2, world=1)
    assert t == 250.0 and v == pytest.approx(8.0)


def _shard_rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    from gpujachx_b200 import batch
    sizes = bench.batch_sizes(4096, 5000)
    parts = batch.partition(sizes, sizes, world)
    mine = parts[rank]
    # every rank computes the same partition; gather the shards to check
    counts = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(counts, torch.tensor([len(mine)]))
    total = torch.zeros(1, dtype=torch.float64)
    dist.all_reduce(total.add_(float(sum(int(x) for x in mine))))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, [int(c) for c in counts], float(total), mine.tolist(), batch.imbalance(parts, sizes, sizes)))


def test_batch_shards_over_two_gloo_ranks():
    """The C5 batch split over 2 ranks by the size-balanced partition: the
    shards are disjoint, cover the batch, and carry equal work within 0.1 %."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31500 + (os.getpid() % 2000)
    ps = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    got = sorted(q.get(timeout=10) for _ in range(2))
    for p in ps:
        assert p.exitcode == 0
    (_, c0, s0, m0, imb), (_, c1, s1, m1, _) = got
    assert c0 == c1 and sum(c0) == 4096
    assert s0 == s1 == float(sum(range(4096)))
    assert not set(m0) & set(m1) and len(set(m0) | set(m1)) == 4096
    assert imb < 1.001


def _shard_data_rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    sizes = bench.batch_sizes(96, 5000)               # the c5 size distribution, a small batch
    offs = np.concatenate([[0], np.cumsum(sizes.astype(np.int64) ** 2)])
    G_all = torch.arange(int(offs[-1]), dtype=torch.float64)   # every element its own index
    mine, sz, soffs, G = bench.shard_batch(G_all, offs, sizes, rank, world)
    parts = [None] * world
    dist.all_gather_object(parts, (mine.tolist(), sz.tolist(), soffs.tolist(), G.numpy()))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put((sizes.tolist(), offs.tolist(), parts))


def test_sharded_batch_reassembles_over_two_gloo_ranks():
    """bench.py --shard: each rank slices its shard out of the same batch;
    the shards are disjoint, cover the batch, and their buffers put back in
    index order give the batch buffer bit for bit."""
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 33600 + (os.getpid() % 2000)
    ps = [ctx.Process(target=_shard_data_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    sizes, offs, parts = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    idx = sorted(i for mine, *_ in parts for i in mine)
    assert idx == list(range(len(sizes)))             # disjoint and complete
    whole = np.empty(offs[-1])
    for mine, sz, soffs, G in parts:
        assert sz == [sizes[i] for i in mine]
        assert soffs[-1] == len(G)
        for k, b in enumerate(mine):
            whole[offs[b]:offs[b + 1]] = G[soffs[k]:soffs[k + 1]]
    assert np.array_equal(whole, np.arange(offs[-1], dtype=np.float64))
    loads = [sum(s * s * s for s in sz) for _, sz, _, _ in parts]
    assert max(loads) / (sum(loads) / 2) < 1.05       # balanced by work
