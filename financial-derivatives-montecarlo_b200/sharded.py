"""Replica and option sharding across ranks (one process per GPU, torch.distributed).

The RQMC estimator is a mean over R independently scrambled replicas, and a book is a list of
independent options, so the path shards without any exchange inside a pass:

* `run_qmc_sharded` — the doubling loop of run_qmc_cuda (methods_cuda.cu:1624-1668) with the R
  replicas split into contiguous blocks, one per rank (replica r keeps salt salt_base + r, so the
  points are those of the one-process run).  After each doubling the per-replica sums are
  exchanged with one all-reduce of an [R][2] FP64 tensor in which every slot has exactly one
  non-zero contributor, so the reduced sums are the per-replica sums bit for bit and every rank
  takes the same stopping decision.
* `price_book_sharded` — options dealt round-robin by index; each rank prices its share with the
  batched book and the results are gathered back into book order.

The compute is passed in as a function, so the same host logic runs on GPUs (NCCL, the engine's
passes) and in the CPU tests (gloo, the oracle).
"""
import math

import torch
import torch.distributed as dist


def _world(group=None):
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def replica_block(R, world, rank):
    """Contiguous replica block [r0, r1) of `rank` among `world` ranks (sizes differ by <= 1)."""
    if R < 1 or world < 1 or not 0 <= rank < world:
        raise ValueError("need R >= 1, world >= 1 and 0 <= rank < world")
    return R * rank // world, R * (rank + 1) // world


def run_qmc_sharded(pass_fn, R, eps, N0, max_doublings=20, group=None, device="cpu"):
    """Adaptive RQMC over R replicas split across the ranks of `group`.

    pass_fn(r0, nr, offset, n) returns the [nr][2] sums {sum Y, sum Y^2} of replicas r0..r0+nr-1
    over points offset..offset+n-1 (an empty block is never asked for).  Returns the dict of
    run_qmc_cuda: price (mean of the replica means), std_error (sqrt of their variance / R),
    n_samples (R N), plus the doublings taken.
    """
    rank, world = _world(group)
    r0, r1 = replica_block(R, world, rank)
    acc = torch.zeros((R, 2), dtype=torch.float64, device=device)
    n_per, done = int(N0), 0
    vom, price, total, dbl = math.inf, 0.0, 0, 0
    for dbl in range(max_doublings):
        if n_per > done:
            part = torch.zeros((R, 2), dtype=torch.float64, device=device)
            if r1 > r0:
                s = pass_fn(r0, r1 - r0, done, n_per - done)
                part[r0:r1] = torch.as_tensor(s, dtype=torch.float64, device=device).reshape(r1 - r0, 2)
            if world > 1:
                dist.all_reduce(part, op=dist.ReduceOp.SUM, group=group)
            acc += part
            done = n_per
        means = (acc[:, 0] / n_per).cpu().tolist()
        mm = 0.0
        for v in means:
            mm += v
        mm /= R
        var = 0.0
        for v in means:
            var += (v - mm) * (v - mm)
        var = var / (R - 1) if R > 1 else 0.0
        vom, price, total = var / R, mm, R * n_per
        if vom < eps * eps / 2.0:
            break
        n_per *= 2
    return {"price": price, "std_error": math.sqrt(vom), "n_samples": total, "doublings": dbl + 1}


def book_share(n_options, world, rank):
    """Indices of the options `rank` prices: i = rank, rank + world, ..."""
    return list(range(rank, n_options, world))


def price_book_sharded(price_fn, options, group=None):
    """Prices a book with its options dealt round-robin over the ranks.

    price_fn(list_of_options) returns one result per option (the batched book on this rank's
    GPU).  Every rank returns the full list of results in book order."""
    rank, world = _world(group)
    mine = book_share(len(options), world, rank)
    res = price_fn([options[i] for i in mine]) if mine else []
    if len(res) != len(mine):
        raise RuntimeError("price_fn returned %d results for %d options" % (len(res), len(mine)))
    if world == 1:
        return list(res)
    parts = [None] * world
    dist.all_gather_object(parts, list(zip(mine, res)), group=group)
    out = [None] * len(options)
    for part in parts:
        for i, r in part:
            out[i] = r
    return out
