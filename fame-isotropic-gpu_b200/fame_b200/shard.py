"""k-point sharding across ranks, one process per GPU.

Wave vectors are independent (the reference's k-loop, FAME_Main/FAME_Main_Code.cu:79-133,
carries no state from one k to the next), so the band path splits into contiguous
blocks, one per rank, with no exchange inside a solve.  The only collective is one
gather of the per-k results (nwant frequencies, residuals and counters per k) after
every rank has solved its block.  Works over any torch.distributed backend (NCCL
between GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_bounds(nk: int, world_size: int, rank: int) -> tuple[int, int]:
    """[start, stop) of rank's contiguous block; block sizes differ by at most one."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("bad rank / world size")
    return nk * rank // world_size, nk * (rank + 1) // world_size


def balanced_bounds(costs, world_size: int) -> list[tuple[int, int]]:
    """Contiguous blocks [start, stop), one per rank, cut where the running sum of the
    per-k costs crosses r / world_size of the total (each cut at the nearer side of the
    crossing), so no block exceeds its share by more than one k-point's cost.  Uniform
    costs give blocks whose sizes differ by at most one.  Costs are e.g. a previous solve's CG iterations per
    k-point (the work of a k-point is its CG iterations times the operator cost, which is
    the same for every k-point of a grid)."""
    c = np.asarray(costs, dtype=np.float64).reshape(-1)
    if world_size < 1 or np.any(c < 0):
        raise ValueError("bad world size or negative cost")
    nk = c.size
    if nk == 0 or not np.any(c > 0):
        return [shard_bounds(nk, world_size, r) for r in range(world_size)]
    pre = np.concatenate([[0.0], np.cumsum(c)])
    tot = pre[-1]
    cuts = [0]
    for r in range(1, world_size):
        t = tot * r / world_size
        i = int(np.searchsorted(pre, t))  # pre[i-1] < t <= pre[i]
        i = min(max(i, 1), nk)
        if t - pre[i - 1] < pre[i] - t:
            i -= 1
        cuts.append(max(cuts[-1], min(i, nk)))
    cuts.append(nk)
    return [(cuts[r], cuts[r + 1]) for r in range(world_size)]


def solve_sharded(ctx, kpoints, params, group=None, resabs=False, costs=None):
    """Solves this rank's block of `kpoints` (nk, 3) on its own context and gathers
    every block to every rank.  Returns dict(freq, relres, relerr, counters[, resabs])
    for all nk k-points in input order.  costs (nk values, or None for equal costs)
    balance the blocks (balanced_bounds).  Without an initialised process group it
    solves everything locally."""
    import torch.distributed as dist

    k = np.asarray(kpoints, dtype=np.float64).reshape(-1, 3)
    nk = k.shape[0]
    if not (dist.is_available() and dist.is_initialized()):
        return ctx.solve(k, params, resabs=resabs)
    ws = dist.get_world_size(group)
    rank = dist.get_rank(group)
    a, b = shard_bounds(nk, ws, rank) if costs is None else balanced_bounds(costs, ws)[rank]
    part = None
    if b > a:
        out = ctx.solve(k[a:b], params, resabs=resabs)
        part = {key: out[key] for key in ("freq", "relres", "relerr", "counters", "resabs") if key in out}
        part["rc"] = out.get("rc", 0)
    parts = [None] * ws
    dist.all_gather_object(parts, (a, b, part), group=group)
    nwant = params.nwant
    res = dict(freq=np.zeros((nk, nwant)), relres=np.zeros((nk, nwant)), relerr=np.zeros((nk, nwant)),
               counters=[None] * nk, rc=0)
    if resabs:
        res["resabs"] = np.zeros((nk, nwant))
    for a_, b_, p in parts:
        if p is None:
            continue
        for key in ("freq", "relres", "relerr") + (("resabs",) if resabs else ()):
            res[key][a_:b_] = p[key]
        res["counters"][a_:b_] = p["counters"]
        res["rc"] = res["rc"] or p["rc"]
    return res
