"""The multi-process path on the CPU: two gloo ranks (world_size 2) shard a
batch of chordal matrices with chompack_b200.shard, compute each share's
log dets (here with the oracle's C restatement, the CPU stand-in for the GPU
sweep), gather them and reduce a timing over ranks.  Every rank must end
with the serial result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from chompack_b200 import shard


def _batch():
    import chompack_b200 as cp
    from chompack_b200 import grids
    rng = np.random.default_rng(3)
    mats = []
    for i, side in enumerate(rng.integers(5, 14, size=7)):
        A = grids.grid2d_extra(int(side), seed=40 + i)
        s = cp.symbolic(A, p=cp.amd.order(A))
        mats.append((A, s))
    return mats


def _logdet_oracle(A, s):
    import chompack_b200 as cp
    from oracle import oracle
    x = (cp.cspmatrix(s, device="cpu") + A).blkval.numpy().copy()
    assert oracle.cholesky(s, x) == 0
    ld = 0.0
    for k in range(s.Nsn):
        nn = int(s.snptr[k + 1] - s.snptr[k])
        nj = int(s.sncolptr[k + 1] - s.sncolptr[k])
        blk = x[int(s.blkptr[k]):int(s.blkptr[k + 1])].reshape((nj, nn), order="F")
        ld += 2.0 * float(np.sum(np.log(np.diag(blk[:nn]))))
    return ld


def _worker(rank, world, port, root, q):
    import sys
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mats = _batch()
        costs = [shard.cholesky_flops(s) for _, s in mats]
        mine = shard.my_share(costs)
        vals = [_logdet_oracle(*mats[i]) for i in mine]
        full = shard.gather_results(mine, vals, len(mats))
        tmax = shard.max_over_ranks(1.0 + rank)
        tsum = shard.sum_over_ranks(float(len(mine)))
        q.put((rank, mine, full, tmax, tsum))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_is_a_balanced_cover():
    costs = [5.0, 1.0, 1.0, 4.0, 3.0, 3.0, 2.0]
    shares = shard.partition(costs, 2)
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in shares]
    assert abs(loads[0] - loads[1]) <= max(costs)
    assert shard.partition(costs, 1) == [list(range(len(costs)))]


def test_two_gloo_ranks_shard_a_batch():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, root, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mats = _batch()
    serial = [_logdet_oracle(A, s) for A, s in mats]
    shares = sorted(r[1] for r in results)
    assert sorted(i for s in shares for i in s) == list(range(len(mats)))   # disjoint cover
    for rank, mine, full, tmax, tsum in results:
        assert full == pytest.approx(serial, rel=1e-13)
        assert tmax == 2.0
        assert tsum == float(len(mats))


def _worker_uneven(rank, world, port, root, q):
    """The benchmark's sharded batch flow (bench.py batch_section) on gloo:
    the uneven grids of grids.uneven_batch_specs (here 12 small ones),
    shares by cholesky flops, per-matrix log dets gathered, the per-rank
    breakdown exchanged with all_gather_object and the time reduced as the
    max over ranks."""
    import sys
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import torch.distributed as dist
    import chompack_b200 as cp
    from chompack_b200 import grids
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = grids.uneven_batch_specs(count=12, lo=6, hi=14)
        mats = []
        for sd, seed in specs:
            A = grids.grid2d_extra(sd, seed=seed)
            mats.append((A, cp.symbolic(A, p=cp.amd.order(A))))
        costs = [shard.cholesky_flops(s) for _, s in mats]
        mine = shard.my_share(costs, rank, world)
        lds = [_logdet_oracle(*mats[i]) for i in mine]
        all_ld = shard.gather_results(mine, lds, len(mats))
        per_rank = [None] * world
        dist.all_gather_object(per_rank, {"rank": rank, "matrices": len(mine)})
        t_max = shard.max_over_ranks(0.5 * (rank + 1))
        q.put((rank, mine, all_ld, per_rank, t_max))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_uneven_batch_like_the_benchmark():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_uneven, args=(r, 2, port, root, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import chompack_b200 as cp
    from chompack_b200 import grids
    serial = []
    for sd, seed in grids.uneven_batch_specs(count=12, lo=6, hi=14):
        A = grids.grid2d_extra(sd, seed=seed)
        serial.append(_logdet_oracle(A, cp.symbolic(A, p=cp.amd.order(A))))
    assert sorted(i for r in results for i in r[1]) == list(range(12))
    for rank, mine, all_ld, per_rank, t_max in results:
        assert all_ld == pytest.approx(serial, rel=1e-13)
        assert [d["rank"] for d in per_rank] == [0, 1]
        assert sum(d["matrices"] for d in per_rank) == 12
        assert t_max == 1.0
