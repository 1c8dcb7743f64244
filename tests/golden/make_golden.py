"""Generates the golden fixtures in tests/golden/ from the reference's own build.

    python tests/golden/make_golden.py pre [NAME ...] # CPU, needs the reference sources
    python tests/golden/make_golden.py ref OUTDIR     # on a B200, runs the reference's
                                                      # FP64 CUDA solver (oracle/_ref)
    python tests/golden/make_golden.py condense OUTDIR
    python tests/golden/make_golden.py ref-big OUTDIR       # on a B200: full-size runs
    python tests/golden/make_golden.py condense-big OUTDIR
    python tests/golden/make_golden.py ref-path OUTDIR      # on a B200: general-lattice paths
    python tests/golden/make_golden.py condense-path OUTDIR
    python tests/golden/make_golden.py ref-adjoint OUTDIR   # on a B200: adjoint config
    python tests/golden/make_golden.py condense-adjoint OUTDIR
    python tests/golden/make_golden.py gamma-oracle         # CPU: hex36 Gamma spectrum
    python tests/golden/make_golden.py hex36-oracle         # CPU: hex36 off-Gamma oracle solves

`pre` runs the reference's preprocessing (FAME_Preprocessing) through
oracle/_ref/fame_ref_harness for every named workload and stores its integer and
geometric outputs (grid, m1-m4, Omega, k path, Binout, ...) as <name>_pre.npz.

`ref` runs the reference's FP64 solver on the small workloads and on the full 96^3
metric band path, writing <name>_ref.jsonl (frequencies, counters, wall time per k)
and <name>_apply.npz (reference Qr/Qrs/QBQ/invAr applied to seeded vectors) into
OUTDIR; `condense OUTDIR` then writes the committed subset into tests/golden/.
`ref-big` runs the full-size configurations (BIG_RUNS): the 96^3 band path at the
reference's default tolerance 1e-12 and a few k-points of FCC 64, BCC 48 and hex
128; `condense-big` writes their frequency and counter fixtures.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_inputs as ri  # noqa: E402

GOLDEN = os.path.dirname(os.path.abspath(__file__))

PRE_NAMES = ["sc16", "sc32", "sc96", "fcc16", "fcc64", "bcc12", "bcc48", "hex12", "hex36", "hex128"]


def material_dict(name):
    m = ri.WORKLOADS[name][0]()
    nm = m["material_num"]
    r12 = lambda v: [float(f"{float(x):.12f}") for x in v]  # as written to the file
    return dict(
        material_num=nm,
        sphere_num=[sum(1 for s in m["spheres"] if s[0] == k) for k in range(nm)],
        sphere_centers=r12([c for k in range(nm) for s in m["spheres"] if s[0] == k for c in s[1]]),
        sphere_radius=r12([s[2] for k in range(nm) for s in m["spheres"] if s[0] == k]),
        cylinder_num=[sum(1 for s in m["cylinders"] if s[0] == k) for k in range(nm)],
        cylinder_top_centers=r12([c for k in range(nm) for s in m["cylinders"] if s[0] == k for c in s[1]]),
        cylinder_bot_centers=r12([c for k in range(nm) for s in m["cylinders"] if s[0] == k for c in s[2]]),
        cylinder_radius=r12([s[3] for k in range(nm) for s in m["cylinders"] if s[0] == k]),
        lattice_type=m["lattice_type"], const=list(m["const"]))


def do_pre(names=None):
    for name in names or PRE_NAMES:
        with tempfile.TemporaryDirectory() as d:
            ri.make_workdir(name, d)
            p = ri.run_pre(d, os.path.join(d, "pre.bin"))
        binout = p.pop("Binout").astype(np.uint8)
        np.savez_compressed(os.path.join(GOLDEN, f"{name}_pre.npz"),
                            Binout_bits=np.packbits(binout), Binout_len=binout.size,
                            material=json.dumps(material_dict(name)), **p)
        print(name, p["grid_nums"], int(binout.sum()))


# k-point subsets solved by the reference on the GPU: (workload, kidx or None=all, nwant)
REF_RUNS = [
    ("sc16", None),
    ("fcc16", None),
    ("bcc12", None),
    ("hex12", None),
    ("sc32", None),
    ("sc96", None),
]


def do_ref(outdir):
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(1234)
    for name, kidx in REF_RUNS:
        with tempfile.TemporaryDirectory() as d:
            ri.make_workdir(name, d)
            out = os.path.join(outdir, f"{name}_ref.jsonl")
            cmd = [ri.REF_HARNESS, "solve", d, out]
            if kidx:
                cmd += ["--kidx", kidx]
            with open(os.path.join(outdir, f"{name}_ref.log"), "w") as log:
                subprocess.run(cmd, check=True, stdout=log, stderr=subprocess.STDOUT)
            if name.endswith("96") or name == "sc32":
                continue
            g = np.load(os.path.join(GOLDEN, f"{name}_pre.npz"))
            N = int(np.prod(g["grid_nums"]))
            x = rng.standard_normal(5 * N) + 1j * rng.standard_normal(5 * N)
            inp = os.path.join(d, "in.bin")
            x.astype("<c16").tofile(inp)
            outb = os.path.join(d, "apply.bin")
            with open(os.path.join(outdir, f"{name}_apply.log"), "w") as log:
                subprocess.run([ri.REF_HARNESS, "apply", d, inp, outb], check=True,
                               stdout=log, stderr=subprocess.STDOUT)
            raw = np.fromfile(outb, "<f8")
            nk = g["WaveVector"].size // 3
            recs = {}
            p = 0
            for k in range(nk):
                Nd = int(raw[p]); p += 1
                for key, n in (("Qr", 3 * N), ("Qrs", 2 * Nd), ("QBQ", 2 * Nd), ("invAr", 2 * Nd)):
                    v = raw[p:p + 2 * n].view("<c16")
                    p += 2 * n
                    recs[f"{key}_{k}"] = v.copy()
                recs[f"Nd_{k}"] = np.array(Nd)
            np.savez_compressed(os.path.join(outdir, f"{name}_apply.npz"), x=x, **recs)
        print("done", name)




# Full-size runs: the 96^3 band path at the reference's default tolerances
# (1e-12, its Popt.txt) and a few k-points of the FCC 64, BCC 48 and hex 128
# configurations at 1e-10.  (name, fixture name, k indices, tolerance)
BIG_RUNS = [
    ("sc96", "sc96_t12", None, 1e-12),
    ("fcc64", "fcc64", "0,1,2", 1e-10),
    ("bcc48", "bcc48", "0,1,2", 1e-10),
    ("hex128", "hex128", "1,2", 1e-10),
]


def do_ref_big(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name, fix, kidx, tol in BIG_RUNS:
        with tempfile.TemporaryDirectory() as d:
            ri.make_workdir(name, d, es_tol=tol, ls_tol=tol)
            out = os.path.join(outdir, f"{fix}_ref.jsonl")
            cmd = [ri.REF_HARNESS, "solve", d, out]
            if kidx:
                cmd += ["--kidx", kidx]
            with open(os.path.join(outdir, f"{fix}_ref.log"), "w") as log:
                subprocess.run(cmd, check=True, stdout=log, stderr=subprocess.STDOUT)
        print("done", fix, flush=True)


def condense_big(src, dst=GOLDEN):
    meta = open(os.path.join(src, "gpu.txt")).read().strip().splitlines()
    for name, fix, kidx, tol in BIG_RUNS:
        recs = [json.loads(l) for l in open(os.path.join(src, f"{fix}_ref.jsonl"))]
        out = dict(workload=name, device=meta[1].split(",")[0], host_cores=int(meta[2]),
                   note=f"reference FP64 CUDA build (oracle/_ref/fame_ref_harness solve), "
                        f"es_tol=ls_tol={tol:g}, es_maxit=100, ls_maxit=1000",
                   kidx=[int(v) for v in kidx.split(",")] if kidx else None, tol=tol,
                   kpoints=[dict(k=r["k"], wave_vec=r["wave_vec"], Nd=r["Nd"], freq=r["freq"],
                                 ls_iter=r["ls_iter"], es_iter=r["es_iter"], wall_s=r["wall_s"])
                            for r in recs])
        with open(os.path.join(dst, f"{fix}_ref.json"), "w") as f:
            json.dump(out, f, indent=1)


# Band paths of the general lattices at the reference's own path resolution:
# hexagonal 128 with part_num 6 (5 k-points per segment, segment end excluded, on
# Gamma-M, M-K, K-Gamma, Gamma-A: the path's first 20 points) and BCC 48 with
# part_num 16 (15 per segment on Gamma-H, H-N, N-Gamma, Gamma-P: the first 60).
# (name, fixture name, part_num, number of leading path points, tolerance)
PATH_RUNS = [
    ("hex128", "hex128_path", 6, 20, 1e-10),
    ("bcc48", "bcc48_path", 16, 60, 1e-10),
]


def do_ref_path(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name, fix, pn, nk, tol in PATH_RUNS:
        with tempfile.TemporaryDirectory() as d:
            ri.make_workdir(name, d, es_tol=tol, ls_tol=tol, part_num=pn)
            out = os.path.join(outdir, f"{fix}_ref.jsonl")
            cmd = [ri.REF_HARNESS, "solve", d, out, "--kidx", ",".join(str(i) for i in range(nk))]
            with open(os.path.join(outdir, f"{fix}_ref.log"), "w") as log:
                subprocess.run(cmd, check=True, stdout=log, stderr=subprocess.STDOUT)
        print("done", fix, flush=True)


def condense_path(src, dst=GOLDEN):
    meta = open(os.path.join(src, "gpu.txt")).read().strip().splitlines()
    for name, fix, pn, nk, tol in PATH_RUNS:
        recs = [json.loads(l) for l in open(os.path.join(src, f"{fix}_ref.jsonl"))]
        out = dict(workload=name, device=meta[1].split(",")[0], host_cores=int(meta[2]),
                   note=f"reference FP64 CUDA build (oracle/_ref/fame_ref_harness solve), part_num={pn}, "
                        f"first {nk} path points, es_tol=ls_tol={tol:g}, es_maxit=100, ls_maxit=1000",
                   part_num=pn, tol=tol,
                   kpoints=[dict(k=r["k"], wave_vec=r["wave_vec"], Nd=r["Nd"], freq=r["freq"],
                                 ls_iter=r["ls_iter"], es_iter=r["es_iter"], wall_s=r["wall_s"])
                            for r in recs])
        with open(os.path.join(dst, f"{fix}_ref.json"), "w") as f:
            json.dump(out, f, indent=1)


# Adjoint check configuration: simple cubic 32^3, one permittivity per voxel drawn
# uniform in [1, 13] from numpy.random.default_rng(0), 8 bands at k = (0.25, 0, 0)
# (Cartesian, without 2*pi), tolerances 1e-12.
ADJ_SEED, ADJ_K, ADJ_NWANT, ADJ_TOL, ADJ_SAMPLES = 0, (0.25, 0.0, 0.0), 8, 1e-12, 1024


def adjoint_eps(N):
    return np.random.default_rng(ADJ_SEED).uniform(1.0, 13.0, N)


def do_ref_adjoint(outdir):
    """The reference's FP64 solve with the per-voxel permittivity written straight
    into its B (fame_ref_harness --eps) and its eigenvectors saved (--evec)."""
    os.makedirs(outdir, exist_ok=True)
    g = np.load(os.path.join(GOLDEN, "sc32_pre.npz"))
    N = int(np.prod(g["grid_nums"]))
    e = adjoint_eps(N)
    with tempfile.TemporaryDirectory() as d:
        ri.make_workdir("sc32", d, es_tol=ADJ_TOL, ls_tol=ADJ_TOL, nwant=ADJ_NWANT)
        np.concatenate([e, e, e]).astype("<f8").tofile(os.path.join(d, "eps.bin"))
        with open(os.path.join(d, "k.txt"), "w") as f:
            f.write("1\n%.17g %.17g %.17g\n" % ADJ_K)
        with open(os.path.join(outdir, "sc32_adjoint_ref.log"), "w") as log:
            subprocess.run([ri.REF_HARNESS, "solve", d, os.path.join(outdir, "sc32_adjoint_ref.jsonl"),
                            "--k", os.path.join(d, "k.txt"), "--eps", os.path.join(d, "eps.bin"),
                            "--evec", os.path.join(outdir, "sc32_adjoint_evec")],
                           check=True, stdout=log, stderr=subprocess.STDOUT)
    print("done sc32_adjoint", flush=True)


def condense_adjoint(src, dst=GOLDEN):
    """Frequencies and the Hellmann-Feynman gradient from the reference's eigenvectors:
    full per-band sums and norms, and the values at ADJ_SAMPLES seeded voxels."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fame_oracle as fo
    g = np.load(os.path.join(GOLDEN, "sc32_pre.npz"))
    N = int(np.prod(g["grid_nums"]))
    e = adjoint_eps(N)
    B = np.concatenate([e, e, e])
    rec = json.loads(open(os.path.join(src, "sc32_adjoint_ref.jsonl")).readline())
    freq = np.array(rec["freq"])
    E = np.fromfile(os.path.join(src, "sc32_adjoint_evec_k000.bin"), "<c16").reshape(ADJ_NWANT, 3 * N)
    G = fo.hellmann_feynman_voxel_gradient(E, freq, B, N)
    idx = np.sort(np.random.default_rng(ADJ_SEED + 1).choice(N, ADJ_SAMPLES, replace=False))
    np.savez_compressed(os.path.join(dst, "sc32_adjoint_ref.npz"), freq=freq, idx=idx, grad=G[:, idx],
                        grad_sum=G.sum(axis=1), grad_norm=np.linalg.norm(G, axis=1),
                        es_iter=rec["es_iter"], ls_iter=rec["ls_iter"])


def do_gamma_oracle(name="hex36", nwant=16, seed=7):
    """Spectrum of A_r at the Gamma point of a hexagonal grid from an independent solver.

    ARPACK (scipy eigsh, implicitly restarted Lanczos from a seeded random start) on
    the oracle's A_r^-1, with the oracle's CG at a relative tolerance of 1e-13: the
    nwant smallest eigenvalues of A_r on its N - 1 null-space-free columns, as
    frequencies sqrt(lambda) with their relative residuals ||A_r v - lambda v|| /
    (lambda ||v||).  Beside them, the oracle's restatement of the reference's solver
    (Lanczos started at e_M, FAME_Fast_Algorithms_Isotropic.cu:20-86) on the same
    k-point: whether that start reaches every band of this grid.  Writes
    <name>_gamma_oracle.json; CPU only, about a minute."""
    import scipy.sparse.linalg as sla
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import fame_oracle as fo
    from fixtures import edge_eps, load_pre
    par = load_pre(name)
    B = edge_eps(par)
    kidx = [int(i) for i in np.where(np.linalg.norm(par["kpoints"], axis=1) < 1e-3)[0]]
    k = par["kpoints"][kidx[0]]
    L = fo.lambdas(k, par)
    assert L.Nd == par["N"] - 1
    invB = 1.0 / B
    s = np.concatenate([L.Lq_sqrt, L.Lq_sqrt])
    M = 2 * L.Nd
    ar = lambda x: s * fo.QBQ(s * x, L, invB)
    op = sla.LinearOperator((M, M), dtype=complex,
                            matvec=lambda x: fo.invAr(x, L, invB, 1e-13 * np.linalg.norm(x), 4000))
    rng = np.random.default_rng(seed)
    v0 = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    th, V = sla.eigsh(op, k=nwant, which="LA", v0=v0, ncv=3 * nwant, tol=1e-13)
    order = np.argsort(1.0 / th)
    lam = 1.0 / th[order]
    res = [float(np.linalg.norm(ar(V[:, i]) - l * V[:, i]) / (l * np.linalg.norm(V[:, i])))
           for i, l in zip(order, lam)]
    ref_alg = fo.solve_k(k, par, B, dict(nwant=nwant, nstep=40, tol=1e-10, maxit=100),
                         dict(tol=1e-10, maxit=1000))
    out = dict(workload=name, grid=list(par["grid"]), gamma_kidx=kidx, Nd=int(L.Nd),
               note="ARPACK (scipy eigsh, seeded random start) on the oracle's A_r^-1 at Gamma; "
                    "freq = sqrt of the smallest eigenvalues of A_r, without the two zero bands",
               freq=[float(v) for v in np.sqrt(lam)], relres=res,
               from_e_M=dict(freq=[float(v) for v in ref_alg.freq], es_iter=int(ref_alg.es_iter),
                             restarts=int(ref_alg.restarts), converged=bool(ref_alg.converged)))
    with open(os.path.join(GOLDEN, f"{name}_gamma_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(name, out["freq"], max(res))


def do_hex36_oracle(name="hex36", kidx=(1, 2, 4), nwant=16):
    """The oracle's FP64 solves (the restated reference algorithm: e_M start, CGS
    Lanczos with lock/purge, CG at an absolute 1e-10) of three off-Gamma vertices of the
    hex 36x30x26 path (M, K and A), with their Lanczos counts.  Writes
    <name>_oracle.json; CPU only, about two minutes."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import fame_oracle as fo
    from fixtures import edge_eps, load_pre
    par = load_pre(name)
    B = edge_eps(par)
    recs = []
    for q in kidx:
        r = fo.solve_k(par["kpoints"][q], par, B, dict(nwant=nwant, nstep=40, tol=1e-10, maxit=100),
                       dict(tol=1e-10, maxit=1000))
        assert r.converged and r.Nd == par["N"]
        recs.append(dict(kidx=int(q), wave_vec=[float(v) for v in par["kpoints"][q]],
                         freq=[float(v) for v in r.freq], es_iter=int(r.es_iter), ls_iter=int(r.ls_iter),
                         restarts=int(r.restarts)))
        print(name, q, r.es_iter, r.freq[:4])
    out = dict(workload=name, grid=list(par["grid"]), tol=1e-10, nwant=nwant,
               note="oracle/fame_oracle.py solve_k (FP64 numpy restatement of the reference's solver)",
               kpoints=recs)
    with open(os.path.join(GOLDEN, f"{name}_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)


def condense(src, dst=GOLDEN):
    """Keeps the committed part of a `ref` run: all frequencies and counters, and
    the operator applications at k-points 0 (Gamma) and 1 only."""
    meta = open(os.path.join(src, "gpu.txt")).read().strip().splitlines()
    for name, _ in REF_RUNS:
        recs = [json.loads(l) for l in open(os.path.join(src, f"{name}_ref.jsonl"))]
        out = dict(workload=name, device=meta[1].split(",")[0], host_cores=int(meta[2]),
                   note="reference FP64 CUDA build (oracle/_ref/fame_ref_harness solve), "
                        "es_tol=ls_tol=1e-10, es_maxit=100, ls_maxit=1000",
                   kpoints=[dict(k=r["k"], wave_vec=r["wave_vec"], Nd=r["Nd"], freq=r["freq"],
                                 ls_iter=r["ls_iter"], es_iter=r["es_iter"], wall_s=r["wall_s"])
                            for r in recs])
        with open(os.path.join(dst, f"{name}_ref.json"), "w") as f:
            json.dump(out, f, indent=1)
        ap = os.path.join(src, f"{name}_apply.npz")
        if os.path.exists(ap):
            z = np.load(ap)
            keep = {"x": z["x"]}
            for k in (0, 1):
                for key in ("Qr", "Qrs", "QBQ", "invAr", "Nd"):
                    keep[f"{key}_{k}"] = z[f"{key}_{k}"]
            np.savez_compressed(os.path.join(dst, f"{name}_apply.npz"), **keep)


if __name__ == "__main__":
    if sys.argv[1] == "pre":
        do_pre(sys.argv[2:])
    elif sys.argv[1] == "ref":
        do_ref(sys.argv[2])
    elif sys.argv[1] == "condense":
        condense(sys.argv[2])
    elif sys.argv[1] == "ref-big":
        do_ref_big(sys.argv[2])
    elif sys.argv[1] == "condense-big":
        condense_big(sys.argv[2])
    elif sys.argv[1] == "ref-path":
        do_ref_path(sys.argv[2])
    elif sys.argv[1] == "condense-path":
        condense_path(sys.argv[2])
    elif sys.argv[1] == "ref-adjoint":
        do_ref_adjoint(sys.argv[2])
    elif sys.argv[1] == "condense-adjoint":
        condense_adjoint(sys.argv[2])
    elif sys.argv[1] == "gamma-oracle":
        do_gamma_oracle()
    elif sys.argv[1] == "hex36-oracle":
        do_hex36_oracle()
    else:
        raise SystemExit(__doc__)
