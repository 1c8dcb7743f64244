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


def solve_sharded(ctx, kpoints, params, group=None, resabs=False):
    """Solves this rank's block of `kpoints` (nk, 3) on its own context and gathers
    every block to every rank.  Returns dict(freq, relres, relerr, counters[, resabs])
    for all nk k-points in input order.  Without an initialised process group it
    solves everything locally."""
    import torch.distributed as dist

    k = np.asarray(kpoints, dtype=np.float64).reshape(-1, 3)
    nk = k.shape[0]
    if not (dist.is_available() and dist.is_initialized()):
        return ctx.solve(k, params, resabs=resabs)
    ws = dist.get_world_size(group)
    rank = dist.get_rank(group)
    a, b = shard_bounds(nk, ws, rank)
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
