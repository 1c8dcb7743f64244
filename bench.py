#!/usr/bin/env python
"""Band-structure throughput benchmark (k-points/s) on B200.

Workload: simple cubic lattice a=1, grid 96^3, one dielectric sphere (r=0.25a,
eps=13) in eps=1, 10 bands, Lanczos restart dimension 40, Lanczos and CG
tolerances 1e-12 (the reference's defaults; relative residual of every band
checked <= 1e-6), the reference's default band path GXMGRX|MR with part_num=4
(20 k-points).  The k
path and the material map are the reference preprocessing outputs committed in
tests/golden/sc96_pre.npz (synthetic crystal; no dataset involved).

One step = one full solve of the 20-k path through the device-resident solver
(inputs already in HBM), all 20 k-points as one batch in one CUDA graph.  The
batch's working set (about 55 GB) is far larger than L2 and each step runs >1000
CG iterations, so L2 state between steps is irrelevant (config records "l2").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision mixed|fp64] [--batch B] [--no-fp64] [--no-cpu-baseline]
                  [--mode solve|qbq|locate|lattices] [--workload W] [--nk K] [--tol T] [--no-graph]

--impl reference runs the reference's own FP64 CUDA build (oracle/_ref, compiled
from the reference sources) through its own FAME_Fast_Algorithms_Driver; each
timed step is the whole 20-point path, one k-point at a time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fame-isotropic-gpu_b200"))

METRIC = "k-points/s at 96^3, 10 bands, resid 1e-6: batched FP32 vs plain FP64, 1 B200"
WORKLOAD = "sc96"
NWANT, NSTEP = 10, 40
# the reference's default solver tolerances (its Popt.txt): Lanczos and CG 1e-12
TOLS = dict(es_tol=1e-12, ls_tol=1e-12, es_maxit=100, ls_maxit=1000)


def load_workload():
    z = np.load(os.path.join(ROOT, "tests", "golden", f"{WORKLOAD}_pre.npz"))
    n = int(z["Binout_len"])
    return dict(
        grid=tuple(int(v) for v in z["grid_nums"]), mesh_len=z["mesh_len"], lattice_vec_a=z["lattice_vec_a"],
        simple=bool(int(z["simple"][0])), m=tuple(int(v) for v in z["m"]), t1=z["t"][:3],
        binout=np.unpackbits(z["Binout_bits"])[:n].astype(np.int32), material_num=int(z["material_num"][0]),
        eps_in=z["ele_permitt_in"], eps_out=float(z["ele_permitt_out"][0]),
        kpoints=z["WaveVector"].reshape(-1, 3))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 4 + i and
                          s[4 + i].lower() in ("active", "1", "yes")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_init(backend="nccl", timeout_s=600):
    """One process per GPU (torchrun sets RANK / LOCAL_RANK / WORLD_SIZE / MASTER_*).
    The process-group timeout bounds every collective, so ranks that wait for a
    rank that has failed end with an error instead of hanging."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws == 1:
        return 0, 1, 0, None
    import datetime
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, ws, local, dist


def max_over_ranks(x, dist):
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def rank_kpoints(W, rank):
    """Weak scaling: every rank solves a 20-point path; rank r's copy is shifted by
    r*1e-3 (Cartesian, no 2*pi) so that ranks solve distinct k-points of equal cost."""
    k = W["kpoints"].copy()
    if rank:
        k = k + 1e-3 * rank
    return k


def cpu_baseline(W, counters):
    """The plain FP64 method on the host cores: oracle/fame_cpu.cpp (the C++/OpenMP
    restatement of the reference's Lanczos / CG / FFT operator, all host threads).
    Measured end to end on the two small simple-cubic workloads (SC 16^3: two
    k-points of its path, 10 bands; SC 32^3 with the 96^3 material: k = (0.25, 0, 0),
    8 bands; tolerance 1e-10).  At 96^3 the time of one CG iteration and of one
    Lanczos step (j = 25) are measured and scaled by the counters of the FP64 solve
    (CG iterations, Lanczos steps per k-point): the `value`, labelled extrapolated."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import fame_cpu as fc
    from fixtures import edge_eps as fx_edge_eps, load_pre
    cores = fc.threads()
    cpu = ""
    try:
        with open("/proc/cpuinfo") as f:
            cpu = next((l.split(":", 1)[1].strip() for l in f if l.startswith("model name")), "")
    except OSError:
        pass
    measured = {}
    p16 = load_pre("sc16")
    walls = []
    for _ in range(3):  # median of 3 runs (solve only; preprocessing is the fixture)
        o = fc.solve(p16, fx_edge_eps(p16), p16["kpoints"][1:3], 10, 40, 1e-10, 100, 1e-10, 1000)
        walls.append(float(np.sum(o["wall_s"])))
    measured["sc16_2k"] = {"kpoints_per_s": round(2 / float(np.median(walls)), 4), "runs": 3,
                           "es_iter": [int(v) for v in o["es_iter"]], "ls_iter": [int(v) for v in o["ls_iter"]]}
    p32 = load_pre("sc32")
    walls = []
    for _ in range(3):
        o = fc.solve(p32, fx_edge_eps(p32), [[0.25, 0.0, 0.0]], 8, 40, 1e-10, 100, 1e-10, 1000)
        walls.append(float(np.sum(o["wall_s"])))
    measured["sc32_1k"] = {"kpoints_per_s": round(1 / float(np.median(walls)), 4), "runs": 3,
                           "es_iter": int(o["es_iter"][0]), "ls_iter": int(o["ls_iter"][0])}
    N = int(np.prod(W["grid"]))
    B = edge_eps(W, N)
    par = dict(grid=W["grid"], mesh_len=W["mesh_len"], lattice_vec_a=W["lattice_vec_a"], simple=True)
    t_cg, t_lz = fc.time_blocks(par, B, W["kpoints"][1], iters=10, jstep=25)
    per_k = [c["ls_iter"] * t_cg + c["es_iter"] * t_lz for c in counters]
    value = len(per_k) / float(np.sum(per_k))
    return {"value": value, "unit": "k-points/s", "cores": cores, "kind": "port", "cpu_model": cpu,
            "extrapolated": True, "measured": measured,
            "sample": f"oracle/fame_cpu.cpp (C++/OpenMP FP64 plain method, {cores} threads): at 96^3 "
                      f"{t_cg:.4f} s per CG iteration and {t_lz:.4f} s per Lanczos step, times the FP64 solve's "
                      f"{int(sum(c['ls_iter'] for c in counters))} CG iterations and "
                      f"{int(sum(c['es_iter'] for c in counters))} Lanczos steps over {len(per_k)} k-points "
                      "(extrapolated; restart rotations not counted); end-to-end solves of SC16 and SC32 in "
                      "`measured`"}


def solve_bytes(counters, N, nwant, nstep, mixed):
    """Algorithmic HBM bytes of a band solve, summed from its per-k counters: every
    FP32 (mixed) or FP64 CG iteration moves B_QBQ + 7M.s (operator: x in, the field out
    of Q_r and into Q_r^*, y out, 1/eps; CG vectors: read r, p, x, Ap, write x, r, p),
    every FP64 refinement step B_QBQ(FP64) + 3M.16, Lanczos step j 4M.16 + 2(j+1)M.16
    (the CGS pass reads U twice), every restart (nstep + 1 + nwant + 1)M.16 (U times the
    rotation), and the restoration nwant(M + 6N).16, with M = 2N complex values per
    reduced vector, s = 8 (FP32) or 16 bytes per complex value.  Lanczos step t of a k
    has j = t for t < nstep and j = nwant + (t - nstep) mod (nstep - nwant) after a
    restart."""
    M = 2 * N

    def qbq(s, r):
        return (2 * M + 6 * N) * s + 3 * N * r

    s, r = (8, 4) if mixed else (16, 8)
    total = 0
    for c in counters:
        b = c["ls_iter"] * (qbq(s, r) + 7 * M * s)
        if mixed:
            b += c.get("refine", 0) * (qbq(16, 8) + 3 * M * 16)
        js = sum(1 + (t if t < nstep else nwant + (t - nstep) % (nstep - nwant)) for t in range(c["es_iter"]))
        b += c["es_iter"] * 4 * M * 16 + 2 * js * M * 16
        b += c.get("restarts", 0) * (nstep + 1 + nwant + 1) * M * 16
        b += nwant * (M + 6 * N) * 16
        total += b
    return total


def bench_config(nk, ws):
    """The workload of a bench line, the same dict in both arms."""
    return {"workload": "SC a=1, 96^3, sphere r=0.25 eps=13 in eps=1, 10 bands, nstep 40, "
                        f"tol {TOLS['es_tol']:g}, path GXMGRX|MR part_num=4",
            "grid": [96, 96, 96], "kpoints_per_gpu": nk, "nwant": NWANT, "nstep": NSTEP,
            "parallelism": f"k-sharding x{ws}"}


def run_ours(args):
    import torch
    import fame_b200 as fb
    rank, ws, local, dist = dist_init()
    torch.cuda.set_device(local)
    W = load_workload()
    ctx = fb.Context(W["grid"], W["mesh_len"], W["lattice_vec_a"], W["simple"], W["m"], W["t1"], device=local)
    ctx.set_material(W["binout"], W["material_num"], W["eps_in"], W["eps_out"])
    N = int(np.prod(W["grid"]))
    kp = rank_kpoints(W, rank)
    if args.nk:
        kp = kp[: args.nk]
    nk = kp.shape[0]
    prec = fb.MIXED if args.precision == "mixed" else fb.FP64
    # the FFT plan autotuner (fame_tune) on this grid and batch, before anything is timed
    plan = ctx.tune(W["kpoints"][1], prec, batch=min(args.batch or nk, 64)) if not args.option else "options"
    apply_options(ctx, args)
    params = fb.solver_params(nwant=NWANT, nstep=NSTEP, precision=prec, batch=args.batch,
                              use_graph=0 if args.no_graph else 1, **TOLS)
    stream = torch.cuda.ExternalStream(ctx.stream())
    out = None
    strong = args.scaling == "strong"
    costs = None
    if strong:
        # strong scaling: the one 20-point path split over the ranks (fame_b200.shard),
        # blocks balanced by each k-point's CG iterations in the first warm-up solve
        from fame_b200.shard import solve_sharded
        kp = W["kpoints"][: args.nk] if args.nk else W["kpoints"]
        nk = kp.shape[0]
        run = lambda: solve_sharded(ctx, kp, params, costs=costs)
    else:
        run = lambda: ctx.solve(kp, params)
    for w in range(args.warmup):
        out = run()
        if strong and w == 0:
            costs = [c["ls_iter"] for c in out["counters"]]
    barrier(dist)
    torch.cuda.synchronize()
    l0 = ctx.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            out = run()
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier(dist)
    dt = ev0.elapsed_time(ev1) / 1e3
    launches = ctx.launch_count() - l0
    T = max_over_ranks(dt, dist)
    value = nk * (1 if strong else ws) * args.steps / T
    # ---- end to end through the public API: host eps -> device, solve, host results
    B_host = edge_eps(W, N)
    e2e_steps = max(1, min(args.steps, 2))
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.set_eps(B_host)
        out_e2e = run()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0, dist)
    e2e = {"value": nk * (1 if strong else ws) * e2e_steps / t_e2e, "unit": "k-points/s", "h2d_bytes_per_step": int(B_host.nbytes + kp.nbytes),
           "d2h_bytes_per_step": int(3 * nk * NWANT * 8 + nk * 24), "steps": e2e_steps}
    # ---- accuracy of this run
    relres_max = float(np.max(out["relres"]))
    fr = out["freq"]
    ref_err = None
    # reference frequencies at the same tolerance when a fixture exists for it
    refp = os.path.join(ROOT, "tests", "golden", f"{WORKLOAD}_t12_ref.json" if TOLS["es_tol"] == 1e-12
                        else f"{WORKLOAD}_ref.json")
    if rank == 0 and os.path.exists(refp):
        ref = json.load(open(refp))
        rf = np.array([r["freq"] for r in ref["kpoints"]])[: fr.shape[0]]
        nz = rf > 0
        ref_err = float(np.max(np.abs(fr[nz] - rf[nz]) / rf[nz]))
    counters = out["counters"]
    es_mean = float(np.mean([c["es_iter"] for c in counters]))
    ls_sum = int(sum(c["ls_iter"] for c in counters))
    # ---- roofline of the dominant kernel: one Q_r^* B^-1 Q_r apply (3 fused stages)
    # to a batch of nb k-points, the batch the solve above ran (automatic: all of them)
    hbm, src = peaks()
    kq = W["kpoints"][1]
    nb = min(args.batch or nk, 64)
    ms, stages = ctx.bench_qbq(kq, prec, reps=10, nbatch=nb)
    s = 8 if prec == fb.MIXED else 16
    r = 4 if prec == fb.MIXED else 8
    alg = nb * ((2 * 2 * N + 6 * N) * s + 3 * N * r)  # B_QBQ = (2M + 6N)s + 3N r per k-point
    achieved = alg / (ms * 1e-3) / 1e9
    stage_bytes = [nb * (2 * N + 3 * N) * s, nb * (6 * N * s + 3 * N * r), nb * (3 * N + 2 * N) * s]
    traffic = None
    tp = os.path.join(ROOT, "profiles", "qbq_96cubed_traffic.json")
    if os.path.exists(tp):
        tj = json.load(open(tp)).get("fp32" if prec == fb.MIXED else "fp64")
        if tj and tj.get("grid") == list(W["grid"]):
            traffic = int(nb * tj["dram_bytes_per_kpoint"])
    roof = {"bound": "hbm", "kernel": f"QBQ apply = plane_inv + pencil + plane_fwd over a batch of {nb} k-points",
            "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
            "peak_source": src, "traffic": traffic, "algorithmic_bytes": alg, "batch": nb,
            "ms_per_launch": round(ms, 5), "us_per_kpoint": round(ms * 1e3 / nb, 2),
            "stage_ms": [round(x, 5) for x in stages],
            "stage_GBps": [round(b / (t * 1e-3) / 1e9, 1) for b, t in zip(stage_bytes, stages)],
            "l2": "flushed (256 MiB write) before every launch"}
    # ---- the dominant work of the mixed solve: one FP32 CG iteration (3 fused kernels)
    # on a batch of nb k-points; the line's `roofline` is this one, the QBQ apply beside it
    if prec == fb.MIXED:
        roof_qbq = roof
        msc, stc = ctx.bench_cg(kq, reps=10, nbatch=nb)
        algc = nb * cg_iter_bytes(N)
        ach = algc / (msc * 1e-3) / 1e9
        trc = None
        tp = os.path.join(ROOT, "profiles", "cg_iter_96cubed_traffic.json")
        if os.path.exists(tp):
            tj = json.load(open(tp))
            if tj.get("grid") == list(W["grid"]):
                trc = int(nb * tj["dram_bytes_per_kpoint"])
        roof = {"bound": "hbm", "kernel": f"FP32 CG iteration = plane_inv<IN_CG> + pencil<PEN_QBQ_CG> + "
                                          f"plane_fwd<EPI_CGR> + cg_decide over a batch of {nb} k-points",
                "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s", "frac": round(ach / hbm, 4),
                "peak_source": src, "traffic": trc, "algorithmic_bytes": algc, "batch": nb,
                "ms_per_launch": round(msc, 5), "us_per_kpoint": round(msc * 1e3 / nb, 2),
                "stage_ms": [round(x, 5) for x in stc],
                "stage_GBps_moved": [round(nb * b / (t * 1e-3) / 1e9, 1) for b, t in zip(cg_stage_bytes(N), stc)],
                "l2": "flushed (256 MiB write) before every iteration", "qbq_apply": roof_qbq}
    # ---- the plain FP64 form on the same path (the metric's comparison): FP64, one
    # k-point at a time (batch 1) as the reference runs it, every k-point of the path,
    # in the CUDA graph; and FP64 batched like the mixed solve, for comparison
    fp64 = None
    fp64_counters = None
    if prec == fb.MIXED and not args.no_fp64:
        def timed_solve(p):
            ctx.solve(kp[:1], p)  # records and instantiates the graph of this configuration
            torch.cuda.synchronize()
            ev0.record(stream)
            o = ctx.solve(kp, p)
            ev1.record(stream)
            ev1.synchronize()
            return o, max_over_ranks(ev0.elapsed_time(ev1) / 1e3, dist)
        p1 = fb.solver_params(nwant=NWANT, nstep=NSTEP, precision=fb.FP64, batch=1, **TOLS)
        o1, t1 = timed_solve(p1)
        pb = fb.solver_params(nwant=NWANT, nstep=NSTEP, precision=fb.FP64, batch=args.batch, **TOLS)
        ob, tb = timed_solve(pb)
        nz = o1["freq"] > 0
        fp64_counters = o1["counters"]
        v1, vb = nk * ws / t1, nk * ws / tb
        fp64 = {"value": v1, "unit": "k-points/s", "batch": 1, "graph": True, "kpoints": nk,
                "speedup_mixed_over_fp64": round(value / v1, 3),
                "max_rel_freq_diff_mixed_vs_fp64": float(np.max(np.abs(fr[nz] - o1["freq"][nz]) / o1["freq"][nz])),
                "max_relres_fp64": float(np.max(o1["relres"])),
                "fp64_ls_iter_total": int(sum(c["ls_iter"] for c in o1["counters"])),
                "batched": {"value": vb, "batch": args.batch or "auto", "graph": True,
                            "speedup_mixed_over_it": round(value / vb, 3)}}
    # ---- the whole solve against HBM: algorithmic bytes from this run's counters
    solve_roof = None
    try:
        sb = solve_bytes(counters, N, NWANT, NSTEP, prec == fb.MIXED)
        t_step = dt / args.steps
        solve_roof = {"bound": "hbm", "algorithmic_bytes_per_step": int(sb), "seconds_per_step": round(t_step, 4),
                      "achieved": round(sb / t_step / 1e9, 1), "peak": hbm, "unit": "GB/s",
                      "frac": round(sb / t_step / 1e9 / hbm, 4),
                      "counts": "CG iterations, FP64 refinements, Lanczos steps, restarts, restoration (bench.solve_bytes)"}
    except (KeyError, TypeError, ValueError, ZeroDivisionError):
        solve_roof = None
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(W, fp64_counters if fp64_counters is not None else counters)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "k-points/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(T / args.steps * 1e3, 2), "higher_is_better": True,
            "scaling": args.scaling, "vs_baseline": None, "dtype": "c64 operator/CG + f64 refinement/Lanczos"
            if prec == fb.MIXED else "f64", "data": "synthetic (reference preprocessing of a synthetic SC crystal)",
            "config": bench_config(nk, ws),
            "run": {"precision": args.precision, "batch": args.batch or "auto", "graph": not args.no_graph,
                    "fft_plan": plan,
                    "lanes": ctx.get_option("lanes") if not args.batch else 1,
                    "l2": "inputs exceed L2 per step (>1000 CG iterations per step)",
                    "vectors": "eigenvalues only (want_vectors 0); the reference arm's timed region also "
                               "restores E and copies it to the host (about 2% of its time)"},
            "accuracy": {"max_relres": relres_max, "max_rel_err_vs_reference_fp64": ref_err,
                         "max_relerr_vs_fp64_rayleigh": float(np.max(out["relerr"]))},
            "counters": {"es_iter_mean": es_mean, "ls_iter_total": ls_sum,
                         "restarts_total": int(sum(c["restarts"] for c in counters)),
                         "fp64_refinements_total": int(sum(c["refine"] for c in counters))},
            "roofline": roof, "solve_roofline": solve_roof, "plain_fp64": fp64, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def cg_iter_bytes(N):
    """Algorithmic bytes of one FP32 CG iteration per k-point, B_QBQ + 7M.s with
    B_QBQ = (2M + 6N).s + 3N.r: the operator's vector in and out, the field out of Q_r
    and into Q_r^* (one read and one write of the 3-component field per 3-D transform),
    1/eps, and the CG vectors (read r, p, x, Ap; write x, r, p), s = 8, r = 4.  The
    kernels move a different set: Ap never reaches memory, but the field makes one
    more round trip between the plane and pencil stages (cg_stage_bytes)."""
    M = 2 * N
    return (2 * M + 6 * N) * 8 + 3 * N * 4 + 7 * M * 8


def cg_stage_bytes(N):
    """Bytes each fused FP32 CG kernel moves per k-point: plane_inv reads r, p, x and
    writes p, x and the 3-component field; the pencil stage reads and writes the field
    and reads 1/eps; plane_fwd reads the field and reads and writes r."""
    M = 2 * N
    return [5 * M * 8 + 3 * N * 8, 6 * N * 8 + 3 * N * 4, 3 * N * 8 + 2 * M * 8]


def apply_options(ctx, args):
    """--option name=value: execution options of the context (fame_set_option)."""
    for o in args.option:
        n, v = o.split("=")
        ctx.set_option(n, int(v))


def run_cg(args):
    """FP32 CG iterations alone (fame_bench_cg, 96^3 or --workload; one k off Gamma
    repeated --batch times), each preceded by a 256 MiB L2 flush: the small case of the
    CG-kernel profiles in profiles/."""
    import fame_b200 as fb
    if args.workload == WORKLOAD:
        W = load_workload()
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from fixtures import load_pre
        W = load_pre(args.workload)
    ctx = fb.Context(W["grid"], W["mesh_len"], W["lattice_vec_a"], W["simple"], W["m"], W["t1"])
    ctx.set_material(W["binout"], W["material_num"], W["eps_in"], W["eps_out"])
    apply_options(ctx, args)
    nb = max(1, args.batch)
    ms, st = ctx.bench_cg(W["kpoints"][1], reps=max(1, args.steps), nbatch=nb)
    N = int(np.prod(W["grid"]))
    hbm, src = peaks()
    gbs = nb * cg_iter_bytes(N) / (ms * 1e-3) / 1e9
    print(json.dumps({"mode": "cg", "workload": args.workload, "grid": list(W["grid"]), "reps": args.steps,
                      "batch": nb, "ms_per_iteration": round(ms, 5), "us_per_kpoint": round(ms * 1e3 / nb, 2),
                      "stage_ms": [round(x, 5) for x in st], "GBps": round(gbs, 1),
                      "frac_of_measured_hbm": round(gbs / hbm, 4), "options": args.option}), flush=True)
    ctx.close()


def run_qbq(args):
    """Q_r^* B^-1 Q_r applies alone (96^3 or --workload; one k off Gamma), each
    preceded by a 256 MiB L2 flush: the small case the kernel profiles in profiles/
    capture."""
    import fame_b200 as fb
    if args.workload == WORKLOAD:
        W = load_workload()
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from fixtures import load_pre
        W = load_pre(args.workload)
    ctx = fb.Context(W["grid"], W["mesh_len"], W["lattice_vec_a"], W["simple"], W["m"], W["t1"])
    ctx.set_material(W["binout"], W["material_num"], W["eps_in"], W["eps_out"])
    prec = fb.MIXED if args.precision == "mixed" else fb.FP64
    k = W["kpoints"][1]
    nb = max(1, args.batch)
    ms, st = ctx.bench_qbq(k, prec, reps=max(1, args.steps), nbatch=nb)
    print(json.dumps({"mode": "qbq", "workload": args.workload, "precision": args.precision,
                      "grid": list(W["grid"]), "reps": args.steps,
                      "batch": nb, "ms_per_launch": round(ms, 5), "us_per_kpoint": round(ms * 1e3 / nb, 2),
                      "stage_ms": [round(x, 5) for x in st]}), flush=True)
    ctx.close()


LATTICES = (("fcc64", 10), ("bcc48", 12), ("hex128", 16))


def run_lattices(args):
    """Band solves of the general-lattice workloads (FCC 64x55x52, BCC 48x45x39,
    hexagonal 128x107x92; the reference's preprocessing outputs in tests/golden/)
    at the tolerance of the reference's runs on the same B200 (1e-10): the non-Gamma
    vertices of each path, mixed precision and FP64, timed with CUDA events on the
    context's stream after a warm-up solve of the same k-points.  The reference's
    k-points/s are its own measured per-k wall times from those runs
    (tests/golden/<name>_ref.json)."""
    import torch
    import fame_b200 as fb
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from fixtures import load_pre, load_ref
    for name, nw in LATTICES:
        par = load_pre(name)
        ref = load_ref(name)
        ctx = fb.Context.from_par(par)
        ctx.set_material(par["binout"], par["material_num"], par["eps_in"], par["eps_out"])
        k = par["kpoints"]
        k = k[np.linalg.norm(k, axis=1) > 0]
        line = {"mode": "lattices", "workload": name, "grid": list(par["grid"]), "nwant": nw, "nk": len(k),
                "tol": ref["tol"],
                "reference_kps": round(len(ref["kpoints"]) / sum(r["wall_s"] for r in ref["kpoints"]), 3)}
        rk = {tuple(np.round(r["wave_vec"], 12)): np.array(r["freq"]) for r in ref["kpoints"]}
        # operator times per k-point (batch 8): the built-in plan, then the tuned one
        kq = k[0]
        line["cg_us_per_kpoint_default_plan"] = round(ctx.bench_cg(kq, reps=5, nbatch=8)[0] * 1e3 / 8, 2)
        line["qbq64_us_per_kpoint_default_plan"] = round(ctx.bench_qbq(kq, fb.FP64, reps=5, nbatch=8)[0] * 1e3 / 8, 2)
        line["fft_plan_fp64"] = ctx.tune(kq, fb.FP64, batch=8)
        line["qbq64_us_per_kpoint_tuned"] = round(ctx.bench_qbq(kq, fb.FP64, reps=5, nbatch=8)[0] * 1e3 / 8, 2)
        line["fft_plan_mixed"] = ctx.tune(kq, fb.MIXED, batch=8)
        line["cg_us_per_kpoint_tuned"] = round(ctx.bench_cg(kq, reps=5, nbatch=8)[0] * 1e3 / 8, 2)
        for prec, tag in ((fb.MIXED, "mixed"), (fb.FP64, "fp64")):
            p = fb.solver_params(nwant=nw, nstep=NSTEP, es_tol=ref["tol"], ls_tol=ref["tol"], es_maxit=100,
                                 ls_maxit=1000, precision=prec)
            ctx.solve(k, p)  # warm-up on the same k-points: lane contexts and graphs exist before timing
            st = torch.cuda.ExternalStream(ctx.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st)
            o = ctx.solve(k, p)
            e1.record(st)
            e1.synchronize()
            line[f"{tag}_kps"] = round(len(k) / (e0.elapsed_time(e1) / 1e3), 3)
            errs = [np.max(np.abs(o["freq"][i] - rk[key]) / rk[key]) for i, key in
                    enumerate(tuple(np.round(v, 12)) for v in k) if key in rk]
            line[f"{tag}_max_rel_diff_vs_reference"] = float(max(errs)) if errs else None
            line[f"{tag}_max_relres"] = float(np.max(o["relres"]))
        print(json.dumps(line), flush=True)
        ctx.close()


def run_locate(args):
    """The material map Binout of the hexagonal 128x107x92 workload: fame_material_locate
    (host in, host out) against the reference's CPU preprocessing, whose time is
    dominated by FAME_Material_Locate_Index (fame_ref_harness pre, the same inputs)."""
    import fame_b200 as fb
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from fixtures import load_pre
    par = load_pre("hex128")
    call = lambda: fb.material_locate(par["grid"], par["mesh_len"], par["lattice_vec_a"], par["Omega"],
                                      par["Permutation"], par["material"])
    for _ in range(max(1, args.warmup)):
        b = call()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps)):
        b = call()
    t = (time.perf_counter() - t0) / max(1, args.steps)
    line = {"mode": "locate", "workload": "hex c/a=1.2, 128x107x92, 2 cylinders r=0.3", "gpu_s": round(t, 5),
            "bit_exact": bool(np.array_equal(b, par["binout"]))}
    harness = os.path.join(ROOT, "oracle", "_ref", "fame_ref_harness")
    if os.path.exists(harness):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ref_inputs as ri
        with tempfile.TemporaryDirectory() as d:
            ri.make_workdir("hex128", d)
            t0 = time.perf_counter()
            subprocess.run([harness, "pre", d, os.path.join(d, "pre.bin")], check=True, stdout=subprocess.DEVNULL)
            line["reference_preprocessing_s"] = round(time.perf_counter() - t0, 3)
    print(json.dumps(line), flush=True)


def edge_eps(W, N):
    """B (3N) from the material map with FAME_Matrix_B_Isotropic's last-wins rule."""
    B = np.full(3 * N, W["eps_out"])
    b = W["binout"].reshape(3, W["material_num"], N)
    for c in range(3):
        for j in range(W["material_num"]):
            B[c * N:(c + 1) * N][b[c, j] == 1] = W["eps_in"][j]
    return B


def run_reference(args):
    """The reference's own FP64 CUDA build (oracle/_ref/fame_ref_harness, compiled from
    the reference sources by oracle/build_ref.sh) through its own preprocessing and
    FAME_Fast_Algorithms_Driver.  Each warm-up step is one k-point; each timed step
    is the whole 20-k band path, one k at a time as the reference runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    harness = os.path.join(ROOT, "oracle", "_ref", "fame_ref_harness")
    if not os.path.exists(harness):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (oracle/build_ref.sh needs the reference sources)"}))
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_inputs as ri
    W = load_workload()
    nkp = W["kpoints"].shape[0]
    if args.nk:
        nkp = min(nkp, args.nk)
    per_step = nkp
    order = [i % nkp for i in range(args.warmup)] + [i for _ in range(args.steps) for i in range(nkp)]
    kidx = ",".join(str(i) for i in order)
    with tempfile.TemporaryDirectory() as d:
        ri.make_workdir(WORKLOAD, d, es_tol=TOLS["es_tol"], es_maxit=TOLS["es_maxit"], ls_tol=TOLS["ls_tol"],
                        ls_maxit=TOLS["ls_maxit"])
        out = os.path.join(d, "out.jsonl")
        with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
            rc = subprocess.run([harness, "solve", d, out, "--kidx", kidx], stdout=subprocess.DEVNULL,
                                stderr=subprocess.PIPE, text=True)
        if rc.returncode != 0:
            print(json.dumps({"impl": "reference", "unavailable": f"reference build failed rc={rc.returncode}: {rc.stderr[-200:]}"}))
            return
        recs = [json.loads(l) for l in open(out)]
    timed = recs[args.warmup:]
    t = sum(r["wall_s"] for r in timed)
    value = len(timed) / t
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "k-points/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t / args.steps * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": bench_config(per_step, int(os.environ.get("WORLD_SIZE", "1"))),
        "run": {"precision": "fp64", "timed_region": "the reference's per-k wall time: its Lanczos solve, its "
                "eigenvector restoration and the D2H copy of E (3N x nwant complex per k)"},
        "cpu_baseline": {"value": round(value, 4), "unit": "k-points/s", "cores": 1, "kind": "reference",
                         "sample": f"{len(timed)} k-points of the 96^3 path through the reference's own FP64 "
                                   "CUDA build (FAME_Fast_Algorithms_Driver; cuFFT/cuBLAS on the B200, one host "
                                   "thread); the reference has no CPU implementation of this path"},
        "e2e": {"value": round(value, 4), "unit": "k-points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_counters": {"es_iter": [r["es_iter"] for r in timed], "ls_iter": [r["ls_iter"] for r in timed]},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="solve", choices=["solve", "qbq", "cg", "locate", "lattices"],
                    help="qbq: only time Q_r^* B^-1 Q_r applies (--steps applies; for kernel profiles); "
                         "lattices: band solves of the FCC, BCC and hexagonal workloads")
    ap.add_argument("--workload", default=WORKLOAD, choices=[WORKLOAD] + [n for n, _ in LATTICES],
                    help="grid of --mode qbq")
    ap.add_argument("--no-graph", action="store_true",
                    help="host-driven loops instead of the CUDA graph (launch lists under ncu)")
    ap.add_argument("--nk", type=int, default=0, help="solve only the first NK k-points (launch-list samples)")
    ap.add_argument("--tol", type=float, default=TOLS["es_tol"], help="Lanczos and CG tolerance")
    ap.add_argument("--option", action="append", default=[], help="execution option name=value (fame_set_option)")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="weak: every rank solves its own 20-point path; strong: the ranks split one path "
                         "(cost-balanced blocks, one gather)")
    args = ap.parse_args()
    TOLS["es_tol"] = TOLS["ls_tol"] = args.tol
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "qbq":
        return run_qbq(args)
    if args.mode == "cg":
        return run_cg(args)
    if args.mode == "locate":
        return run_locate(args)
    if args.mode == "lattices":
        return run_lattices(args)
    return run_ours(args)


if __name__ == "__main__":
    main()
