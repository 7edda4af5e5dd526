"""Multi-GPU sharding of independent work (one process per GPU).

A single chordal matrix is factored on one GPU; what spreads over GPUs is a
batch of independent matrices or value sets.  There is no data exchange on
the sweep path: each rank takes a share of the batch (balanced by estimated
flops, longest first), sweeps it with its own merged plan, and only the
per-matrix results (log dets, timings) are gathered.  Timings are reduced
as the maximum over ranks.

These helpers use torch.distributed (NCCL between GPUs; gloo on the host
for tests).
"""
import torch
import torch.distributed as dist

__all__ = ["partition", "my_share", "max_over_ranks", "sum_over_ranks", "gather_results", "cholesky_flops"]


def cholesky_flops(symb):
    """Algorithmic flops of one cholesky sweep (sum over supernodes of
    nn^3/3 + 2 nn^2 na + nn na^2)."""
    tot = 0.0
    for k in range(symb.Nsn):
        nn = float(symb.snptr[k + 1] - symb.snptr[k])
        na = float(symb.relptr[k + 1] - symb.relptr[k])
        tot += nn ** 3 / 3.0 + 2.0 * nn ** 2 * na + nn * na ** 2
    return tot


def partition(costs, world):
    """Deterministic longest-processing-time assignment of items with the
    given costs to `world` shares: a list of index lists, each in increasing
    order, together covering every item exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    shares = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda w: (load[w], w))
        shares[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in shares]


def my_share(costs, rank=None, world=None):
    """This rank's item indices."""
    if rank is None:
        rank = dist.get_rank() if dist.is_initialized() else 0
    if world is None:
        world = dist.get_world_size() if dist.is_initialized() else 1
    return partition(costs, world)[rank]


def _reduce(value, op, device):
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, device="cpu"):
    """max of a scalar over all ranks (timings: the job ends with the slowest
    rank)."""
    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value, device="cpu"):
    return _reduce(value, dist.ReduceOp.SUM, device)


def gather_results(indices, values, n_items):
    """Assemble per-item results computed on the ranks: every rank passes
    its item indices and values; every rank gets the full list (None where
    no rank supplied a value)."""
    local = list(zip([int(i) for i in indices], [float(v) for v in values]))
    if dist.is_initialized() and dist.get_world_size() > 1:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, local)
    else:
        parts = [local]
    out = [None] * n_items
    for part in parts:
        for i, v in part:
            out[i] = v
    return out
