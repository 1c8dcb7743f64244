"""k-point sharding on two ranks over gloo (CPU, no GPU): fame_b200.shard and the
rank helpers of bench.py.  The solver is a stand-in with a deterministic result
per k-point, so the test covers the partition, the gather in input order, empty
blocks, the max-over-ranks timing reduction, and a rank that fails before the
gather (the other rank's collective ends with an error, not a hang)."""
import json
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

import fame_b200 as fb  # noqa: E402
from fame_b200.shard import balanced_bounds, shard_bounds, solve_sharded  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class FakeCtx:
    """Answers like Context.solve with values that depend only on each k-point."""

    def solve(self, k, params, resabs=False):
        k = np.asarray(k).reshape(-1, 3)
        base = k @ np.array([1.0, 10.0, 100.0])
        freq = base[:, None] + np.arange(params.nwant)[None, :]
        out = dict(freq=freq, relres=freq * 1e-9, relerr=freq * 1e-12, rc=0,
                   counters=[dict(es_iter=int(round(b * 1000)) % 97, ls_iter=7) for b in base])
        if resabs:
            out["resabs"] = freq * 1e-11
        return out


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, outdir, nk, fail_rank, costs=None):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    import bench
    _, _, _, d = bench.dist_init(backend="gloo", timeout_s=20)
    res = {}
    try:
        k = np.random.default_rng(5).uniform(-0.5, 0.5, (nk, 3))
        p = fb.solver_params(nwant=4)
        if rank == fail_rank:
            raise RuntimeError("rank failed before the gather")
        out = solve_sharded(FakeCtx(), k, p, resabs=True, costs=costs)
        ref = FakeCtx().solve(k, p, resabs=True)
        res["freq_ok"] = bool(np.array_equal(out["freq"], ref["freq"]))
        res["resabs_ok"] = bool(np.array_equal(out["resabs"], ref["resabs"]))
        res["counters_ok"] = out["counters"] == ref["counters"]
        res["max"] = bench.max_over_ranks(rank + 1.5, d)
        kr = bench.rank_kpoints(dict(kpoints=k), rank)
        res["rank_k"] = kr[0].tolist()
        bench.barrier(d)
    except Exception as e:  # reported to the parent
        res["error"] = f"{type(e).__name__}: {e}"
    with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)
    if rank == fail_rank:
        os._exit(0)  # leave without joining any further collective
    dist.destroy_process_group()


def _run(tmp_path, nk, fail_rank=-1, ws=2, costs=None):
    mp.spawn(_worker, args=(ws, _free_port(), str(tmp_path), nk, fail_rank, costs), nprocs=ws, join=True)
    return [json.load(open(tmp_path / f"rank{r}.json")) for r in range(ws)]


def test_shard_bounds_cover_every_kpoint_once():
    for nk in (0, 1, 2, 7, 20, 60):
        for ws in (1, 2, 3, 8):
            spans = [shard_bounds(nk, ws, r) for r in range(ws)]
            assert spans[0][0] == 0 and spans[-1][1] == nk
            assert all(spans[i][1] == spans[i + 1][0] for i in range(ws - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def test_two_ranks_gather_in_input_order(tmp_path):
    r0, r1 = _run(tmp_path, nk=7)
    for r in (r0, r1):
        assert "error" not in r, r
        assert r["freq_ok"] and r["resabs_ok"] and r["counters_ok"]
        assert r["max"] == 2.5
    assert r0["rank_k"] != r1["rank_k"]  # weak scaling: each rank solves its own shifted path


def test_fewer_kpoints_than_ranks(tmp_path):
    r0, r1 = _run(tmp_path, nk=1)
    assert r0["freq_ok"] and r1["freq_ok"]


def test_failed_rank_ends_the_other_ranks_collective(tmp_path):
    r0, r1 = _run(tmp_path, nk=6, fail_rank=1)
    assert "rank failed" in r1["error"]
    assert "error" in r0  # the gather saw the lost peer and raised


def test_balanced_bounds_split_by_cost():
    rng = np.random.default_rng(2)
    for nk in (1, 2, 7, 20, 60):
        for ws in (1, 2, 3, 8):
            c = rng.uniform(1.0, 3.0, nk)
            spans = balanced_bounds(c, ws)
            assert spans[0][0] == 0 and spans[-1][1] == nk
            assert all(spans[i][1] == spans[i + 1][0] for i in range(ws - 1))
            share = c.sum() / ws
            assert max(c[a:b].sum() for a, b in spans) <= share + c.max() + 1e-9
    # the reference's pattern on its 20-point 96^3 path: a few k-points need 1.9x the CG work
    cost = np.array([2781, 2820, 2816, 1973, 1976, 1973, 2810, 2813, 1976, 2781,
                     1969, 1966, 1955, 1970, 1972, 1973, 2810, 2813, 3650, 1955], float)
    even = max(cost[a:b].sum() for a, b in (shard_bounds(20, 4, r) for r in range(4)))
    bal = max(cost[a:b].sum() for a, b in balanced_bounds(cost, 4))
    assert bal < even
    sizes = [b - a for a, b in balanced_bounds(np.ones(10), 3)]
    assert sum(sizes) == 10 and max(sizes) - min(sizes) <= 1


def test_two_ranks_gather_with_cost_balanced_blocks(tmp_path):
    costs = [5.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
    r0, r1 = _run(tmp_path, nk=7, costs=costs)
    for r in (r0, r1):
        assert "error" not in r, r
        assert r["freq_ok"] and r["resabs_ok"] and r["counters_ok"]
