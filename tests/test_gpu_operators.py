"""Operator parity on the GPU: the fused sm_100a kernels behind fame_apply against
the reference's FP64 CUDA outputs (tests/golden/*_apply.npz) and the oracle.

Tolerances: FP64 operators within 1e-12 relative (norm-wise) of the reference;
FP32 operators within 1e-5 relative; A_r^-1 (CG to 1e-10 absolute) within 1e-8.
"""
import numpy as np
import pytest

import fame_b200 as fb
import fame_oracle as fo
from fixtures import edge_eps, load_apply, load_pre

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NAMES = ["sc16", "fcc16", "bcc12", "hex12"]


def _ctx(par):
    ctx = fb.Context.from_par(par)
    ctx.set_material(par["binout"], par["material_num"], par["eps_in"], par["eps_out"])
    return ctx


def _run(ctx, op, k, x, n_out, prec=fb.FP64, params=None):
    dt = torch.complex128 if prec == fb.FP64 else torch.complex64
    xd = torch.from_numpy(np.ascontiguousarray(x)).to("cuda", dt)
    yd = torch.zeros(n_out, dtype=dt, device="cuda")
    nd = ctx.apply(op, k, xd, yd, prec, params)
    return yd.cpu().numpy().astype(np.complex128), nd


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("kidx", [0, 1])
def test_fp64_operators_match_reference(name, kidx):
    par = load_pre(name)
    ap = load_apply(name)
    ctx = _ctx(par)
    N = par["N"]
    k = par["kpoints"][kidx]
    Nd = int(ap[f"Nd_{kidx}"])
    x = ap["x"]
    x0 = x[: 2 * Nd]
    v0 = x[2 * N: 5 * N]
    y, nd = _run(ctx, fb.OP_QR, k, x0, 3 * N)
    assert nd == Nd
    assert rel(y, ap[f"Qr_{kidx}"]) < 1e-12
    y, _ = _run(ctx, fb.OP_QRS, k, v0, 2 * Nd)
    assert rel(y, ap[f"Qrs_{kidx}"]) < 1e-12
    y, _ = _run(ctx, fb.OP_QBQ, k, x0, 2 * Nd)
    assert rel(y, ap[f"QBQ_{kidx}"]) < 1e-12
    y, _ = _run(ctx, fb.OP_INVAR, k, x0, 2 * Nd, params=fb.solver_params(ls_tol=1e-10, ls_maxit=1000))
    assert rel(y, ap[f"invAr_{kidx}"]) < 1e-8


@pytest.mark.parametrize("name", NAMES)
def test_fp64_pr_prs_match_oracle(name):
    par = load_pre(name)
    ctx = _ctx(par)
    N = par["N"]
    k = par["kpoints"][1]
    L = fo.lambdas(k, par)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(2 * L.Nd) + 1j * rng.standard_normal(2 * L.Nd)
    v = rng.standard_normal(3 * N) + 1j * rng.standard_normal(3 * N)
    y, _ = _run(ctx, fb.OP_PR, k, x, 3 * N)
    assert rel(y, fo.Pr(x, L)) < 1e-12
    y, _ = _run(ctx, fb.OP_PRS, k, v, 2 * L.Nd)
    assert rel(y, fo.Prs(v, L)) < 1e-12


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("kidx", [0, 2])
def test_fp32_operators_track_fp64(name, kidx):
    par = load_pre(name)
    ctx = _ctx(par)
    N = par["N"]
    k = par["kpoints"][kidx]
    L = fo.lambdas(k, par)
    B = edge_eps(par)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(2 * L.Nd) + 1j * rng.standard_normal(2 * L.Nd)
    v = rng.standard_normal(3 * N) + 1j * rng.standard_normal(3 * N)
    y, _ = _run(ctx, fb.OP_QR, k, x, 3 * N, fb.MIXED)
    assert rel(y, fo.Qr(x, L)) < 1e-5
    y, _ = _run(ctx, fb.OP_QRS, k, v, 2 * L.Nd, fb.MIXED)
    assert rel(y, fo.Qrs(v, L)) < 1e-5
    y, _ = _run(ctx, fb.OP_QBQ, k, x, 2 * L.Nd, fb.MIXED)
    assert rel(y, fo.QBQ(x, L, 1.0 / B)) < 1e-5


def test_metric_grid_qbq_properties():
    """96^3 (the bench grid): Q_r^* Q_r = I and homogeneous-medium QBQ = x / eps."""
    par = load_pre("sc96")
    ctx = fb.Context.from_par(par)
    N = par["N"]
    eps = 4.0
    ctx.set_eps(np.full(3 * N, eps))
    k = par["kpoints"][5]
    rng = np.random.default_rng(3)
    x = rng.standard_normal(2 * N) + 1j * rng.standard_normal(2 * N)
    y, _ = _run(ctx, fb.OP_QR, k, x, 3 * N)
    z, _ = _run(ctx, fb.OP_QRS, k, y, 2 * N)
    assert rel(z, x) < 1e-12
    q, _ = _run(ctx, fb.OP_QBQ, k, x, 2 * N)
    assert rel(q, x / eps) < 1e-12
    q32, _ = _run(ctx, fb.OP_QBQ, k, x, 2 * N, fb.MIXED)
    assert rel(q32, x / eps) < 1e-5


@pytest.mark.parametrize("grid", [(23, 19, 34), (34, 23, 19), (17, 38, 21), (107, 6, 8), (92, 107, 4)])
def test_prime_axis_lengths_match_oracle(grid):
    """Axis lengths with prime factors >= 17 (alone, and after a radix-2 or radix-3
    pass, so the prime pass runs with and without Stockham twiddles) in the plane
    and the pencil stages: a simple-cubic lattice with a random B, FP64 within 1e-12
    and FP32 within 1e-5 of the oracle.  A whole-line prime axis runs in FP32 on the
    tensor cores: 107 points along the fast axis (6 lines per plane) and along the mid
    axis (92 lines per plane: two rounds of line tiles)."""
    N = int(np.prod(grid))
    par = dict(grid=grid, mesh_len=np.array([1.0 / g for g in grid]),
               lattice_vec_a=np.array([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0]), simple=True,
               m=(0, 0, 0, 0), t1=np.zeros(3))
    ctx = fb.Context.from_par(par)
    rng = np.random.default_rng(13)
    B = rng.uniform(1.0, 13.0, 3 * N)
    ctx.set_eps(B)
    k = np.array([0.3, -0.2, 0.45]) * 2 * np.pi
    L = fo.lambdas(k, par)
    x = rng.standard_normal(2 * L.Nd) + 1j * rng.standard_normal(2 * L.Nd)
    v = rng.standard_normal(3 * N) + 1j * rng.standard_normal(3 * N)
    for prec, tol in ((fb.FP64, 1e-12), (fb.MIXED, 1e-5)):
        y, _ = _run(ctx, fb.OP_QR, k, x, 3 * N, prec)
        assert rel(y, fo.Qr(x, L)) < tol
        y, _ = _run(ctx, fb.OP_QRS, k, v, 2 * L.Nd, prec)
        assert rel(y, fo.Qrs(v, L)) < tol
        y, _ = _run(ctx, fb.OP_QBQ, k, x, 2 * L.Nd, prec)
        assert rel(y, fo.QBQ(x, L, 1.0 / B)) < tol
