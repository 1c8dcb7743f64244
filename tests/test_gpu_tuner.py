"""FFT plan autotuner (fame_tune) and the plan options it searches.

Every candidate plan the tuner can pick (radix orders 0..3, plane CTA sizes 128, 256
and 512 threads, in FP64 and FP32) keeps the operator bars against the reference's
FP64 CUDA outputs (tests/golden/*_apply.npz): Q_r^* B^-1 Q_r within 1e-12 relative in
FP64 and 1e-5 in FP32.  fame_tune writes its winner to the cache file, applies a
cached plan without timing, and a solve on the tuned context still matches the
reference's frequencies (mixed precision, 1e-6)."""
import numpy as np
import pytest

import fame_b200 as fb
from fixtures import load_apply, load_pre, load_ref

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _ctx(name):
    par = load_pre(name)
    ctx = fb.Context.from_par(par)
    ctx.set_material(par["binout"], par["material_num"], par["eps_in"], par["eps_out"])
    return par, ctx


def _qbq(ctx, k, x, nd, prec):
    dt = torch.complex128 if prec == fb.FP64 else torch.complex64
    xd = torch.from_numpy(np.ascontiguousarray(x[: 2 * nd])).to("cuda", dt)
    yd = torch.zeros(2 * nd, dtype=dt, device="cuda")
    ctx.apply(fb.OP_QBQ, k, xd, yd, prec)
    return yd.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("name", ["sc16", "fcc16", "bcc12", "hex12"])
def test_every_candidate_plan_keeps_operator_parity(name):
    par, ctx = _ctx(name)
    ap = load_apply(name)
    k = par["kpoints"][1]
    nd = int(ap["Nd_1"])
    ref = ap["QBQ_1"]
    sigs = set()
    for order in range(4):
        try:
            ctx.set_option("radix_order", order)
        except fb.FameError:
            continue  # this order needs a pass level the grid's kernels do not have
        sigs.add(ctx.get_option("plan_signature"))
        for th in (128, 256, 512):
            ctx.set_option("plane_threads64", th)
            ctx.set_option("plane_threads32", th)
            y64 = _qbq(ctx, k, ap["x"], nd, fb.FP64)
            y32 = _qbq(ctx, k, ap["x"], nd, fb.MIXED)
            assert np.linalg.norm(y64 - ref) / np.linalg.norm(ref) < 1e-12, (order, th)
            assert np.linalg.norm(y32 - ref) / np.linalg.norm(ref) < 1e-5, (order, th)
    assert len(sigs) >= 2  # the orders give different plans on these grids
    ctx.close()


def test_tune_caches_and_keeps_the_solve_exact(tmp_path):
    par, ctx = _ctx("fcc16")
    cache = str(tmp_path / "plans.txt")
    k = par["kpoints"][1]
    plan = ctx.tune(k, fb.MIXED, batch=2, cache_file=cache)
    assert "radix_order=" in plan and "(cached)" not in plan
    line = open(cache).read().strip().splitlines()[-1]
    assert line.startswith("grid=16x") and "precision=mixed batch=2 | " in line
    assert ctx.tune(k, fb.MIXED, batch=2, cache_file=cache).endswith("(cached)")
    ref = load_ref("fcc16")
    ks = np.array([r["wave_vec"] for r in ref["kpoints"][:3]])
    out = ctx.solve(ks, fb.solver_params(precision=fb.MIXED, nwant=10, nstep=40, es_tol=1e-10, ls_tol=1e-10))
    for i in range(3):
        rf = np.array(ref["kpoints"][i]["freq"])
        nz = rf > 0
        assert np.max(np.abs(out["freq"][i][nz] - rf[nz]) / rf[nz]) < 1e-6
    ctx.close()
