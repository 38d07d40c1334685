"""Replica and option sharding across ranks (one process per GPU, torch.distributed).

The RQMC estimator is a mean over R independently scrambled replicas, and a book is a list of
independent options, so the path shards without any exchange inside a pass:

* `combine_replica_sums` — the one exchange of a replica-split estimator: each rank's block of
  per-replica sums into the [R][k] sums of all replicas on every rank (one all-reduce, one
  contributor per slot, so bit for bit).  The multi-GPU benchmark uses it after every pass.
* `run_qmc_sharded` — the doubling loop of run_qmc_cuda (methods_cuda.cu:1624-1668) with the R
  replicas split into contiguous blocks, one per rank (replica r keeps salt salt_base + r, so the
  points are those of the one-process run).  After each doubling the per-replica sums are
  exchanged with one all-reduce of an [R][2] FP64 tensor in which every slot has exactly one
  non-zero contributor, so the reduced sums are the per-replica sums bit for bit and every rank
  takes the same stopping decision.
* `run_mlqmc_sharded` — the adaptive MLQMC loop of run_mlqmc_cuda (methods_cuda.cu:1680-2016)
  with every level's R replicas split the same way (replica r of level l keeps salt
  salt_base + l R + r and the level's shared point offsets); each collect is one all-reduce of
  the level's [R][4] sums, every slot with one contributor, so all ranks take the same
  decisions.  With a per-replica pass whose sums do not depend on which other replicas share its
  launch (the oracle in the CPU tests) the result is the one-process result bit for bit; the
  engine's passes split each launch into work items by the launch's size, so on GPUs the sums
  (and, through them, at most the rounding of a sample count) differ from one process's in the
  FP64 summation order only.
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


def combine_replica_sums(local, R, group=None):
    """The estimator's per-replica sums over all ranks of `group`.

    `local` is this rank's [nr][k] tensor of sums for its contiguous replica block
    replica_block(R, world, rank) (nr = its size, 0 allowed).  Returns the [R][k] FP64 tensor, on
    local's device, of every replica's sums on every rank: one all-reduce in which each slot has a
    single non-zero contributor, so each replica's sums arrive bit for bit."""
    rank, world = _world(group)
    r0, r1 = replica_block(R, world, rank)
    local = torch.as_tensor(local, dtype=torch.float64)
    k = local.shape[-1] if local.dim() == 2 else 1
    full = torch.zeros((R, k), dtype=torch.float64, device=local.device)
    if r1 > r0:
        full[r0:r1] = local.reshape(r1 - r0, k)
    if world > 1:
        dist.all_reduce(full, op=dist.ReduceOp.SUM, group=group)
    return full


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
            s = pass_fn(r0, r1 - r0, done, n_per - done) if r1 > r0 else torch.zeros((0, 2))
            acc += combine_replica_sums(torch.as_tensor(s, dtype=torch.float64, device=device).reshape(r1 - r0, 2),
                                        R, group)
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


def run_mlqmc_sharded(level_fn, R, eps, M=2, max_L=10, pilot_n=1000, group=None, device="cpu",
                      max_iter=50):
    """Adaptive MLQMC over R replicas per level, the replicas split across the ranks of `group`.

    level_fn(l, r0, nr, offset, n) returns the [nr][4] sums {sum dY, sum dY^2, sum Yf, sum Yf^2}
    of level l (the coupled fine / coarse pair; level 0 without a coarse path) for replicas
    r0..r0+nr-1 over points offset..offset+n-1 (an empty block is never asked for).  The
    arithmetic is run_mlqmc_cuda's: pilots of pilot_n points on levels 0..2, per level the mean E_l
    of the replica means of dY and sig2_l = their sample variance x N_l, the optimal
    N_l = ceil(2 / (R eps^2) sqrt(sig2_l / M^l) sum_k sqrt(sig2_k M^k)) (at least 100), the merge
    of the extra samples, the bias test max(|E_L|, |E_{L-1}|) / (M - 1) < eps / sqrt(2), a new
    level from its pilot, at most max_iter iterations.  Returns price, std_error, n_samples,
    levels and converged."""
    rank, world = _world(group)
    r0, r1 = replica_block(R, world, rank)
    nl = max_L + 1
    E, sig2, N, off = [0.0] * nl, [0.0] * nl, [0] * nl, [0] * nl

    def collect(l, n):
        s = level_fn(l, r0, r1 - r0, off[l], n) if r1 > r0 else torch.zeros((0, 4))
        part = combine_replica_sums(torch.as_tensor(s, dtype=torch.float64, device=device).reshape(r1 - r0, 4),
                                    R, group)
        off[l] += n
        means = (part[:, 0] / n).cpu().tolist()
        mm = 0.0
        for v in means:
            mm += v
        mm /= R
        var = 0.0
        for v in means:
            var += (v - mm) * (v - mm)
        return mm, (var / (R - 1) if R > 1 else 0.0)

    def absorb(l, n, mv):
        mm, vv = mv
        if N[l] == 0:
            E[l], sig2[l] = mm, vv * n
        else:
            wo, wn = float(N[l]), float(n)
            E[l] = (E[l] * wo + mm * wn) / (wo + wn)
            sig2[l] = (sig2[l] * wo + vv * wn * wn) / (wo + wn)
        N[l] += n

    L = 2
    for l in range(L + 1):
        absorb(l, pilot_n, collect(l, pilot_n))
    converged, it = False, 0
    while not converged and L <= max_L and it < max_iter:
        it += 1
        st = 0.0
        for l in range(L + 1):
            st += math.sqrt(sig2[l] * float(M) ** l)
        extra = []
        for l in range(L + 1):
            nopt = max(int(math.ceil(2.0 / (R * eps * eps) * math.sqrt(sig2[l] / float(M) ** l) * st)), 100)
            extra.append(nopt - N[l] if nopt > N[l] else 0)
        for l in range(L + 1):
            if extra[l] > 0:
                absorb(l, extra[l], collect(l, extra[l]))
        bias = abs(E[L]) / max(M - 1, 1)
        if L >= 1:
            bias = max(bias, abs(E[L - 1]) * M / max(M * (M - 1), 1))
        converged = bias < eps / math.sqrt(2.0)
        if not converged and L < max_L:
            L += 1
            absorb(L, pilot_n, collect(L, pilot_n))
    price, vs = 0.0, 0.0
    for l in range(L + 1):
        price += E[l]
        vs += sig2[l] / (N[l] * R)
    return {"price": price, "std_error": math.sqrt(vs), "n_samples": sum(N[:L + 1]) * R, "levels": L + 1,
            "converged": converged}


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
