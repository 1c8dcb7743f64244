"""Hellmann-Feynman adjoint (fame_adjoint, behind fame_b200.autograd.BandFrequencies)
on the adjoint configuration: simple cubic 32^3, one permittivity per voxel drawn
uniform in [1, 13] (numpy.random.default_rng(0)), 8 bands at k = (0.25, 0, 0),
Lanczos and CG tolerances 1e-12.

Bars:
  * frequencies within 1e-8 (FP64) / 1e-6 (mixed) of the reference's FP64 build run
    on the same permittivity (tests/golden/sc32_adjoint_ref.npz);
  * gradient within 1e-6 (FP64 forward) / 1e-4 (mixed forward) of the FP64 reference
    gradient, the Hellmann-Feynman formula on the reference's own eigenvectors;
  * central finite differences with step 1e-4 along random directions within 1e-4;
  * Euler's identity sum_v eps_v dw/deps_v = -w/2 (w scales as eps^-1/2) within 1e-8;
  * autograd through torch equals the adjoint contraction.
"""
import os

import numpy as np
import pytest

import fame_b200 as fb
from fixtures import GOLDEN, load_pre

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

K = (0.25, 0.0, 0.0)
NWANT = 8
TOLS = dict(nwant=NWANT, nstep=40, es_tol=1e-12, ls_tol=1e-12, es_maxit=100, ls_maxit=1000)


@pytest.fixture(scope="module")
def setup():
    par = load_pre("sc32")
    N = par["N"]
    eps = np.random.default_rng(0).uniform(1.0, 13.0, N)
    ctx = fb.Context.from_par(par)
    ref = np.load(os.path.join(GOLDEN, "sc32_adjoint_ref.npz"))
    return par, ctx, eps, ref


def _solve(ctx, eps, precision=fb.FP64, vectors=True):
    ctx.set_eps(np.concatenate([eps, eps, eps]))
    out = ctx.solve(np.array([K]), fb.solver_params(precision=precision, want_vectors=int(vectors), **TOLS))
    assert out["rc"] == fb.OK
    return out


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b)


@pytest.mark.parametrize("precision,ftol,gtol", [(fb.FP64, 1e-8, 1e-6), (fb.MIXED, 1e-6, 1e-4)])
def test_gradient_matches_reference(setup, precision, ftol, gtol):
    _, ctx, eps, ref = setup
    out = _solve(ctx, eps, precision)
    w = out["freq"][0]
    assert np.max(np.abs(w - ref["freq"]) / ref["freq"]) < ftol
    G = ctx.adjoint(w, out["evec"][0])
    for i in range(NWANT):
        assert _rel(G[i, ref["idx"]], ref["grad"][i]) < gtol
        assert abs(G[i].sum() - ref["grad_sum"][i]) < gtol * abs(ref["grad_sum"][i])


def test_euler_identity(setup):
    _, ctx, eps, _ = setup
    out = _solve(ctx, eps)
    w = out["freq"][0]
    G = ctx.adjoint(w, out["evec"][0])
    np.testing.assert_allclose(G @ eps, -w / 2, rtol=1e-8)


def test_central_differences(setup):
    _, ctx, eps, _ = setup
    out = _solve(ctx, eps)
    G = ctx.adjoint(out["freq"][0], out["evec"][0])
    rng = np.random.default_rng(7)
    h = 1e-4
    for _ in range(3):
        d = rng.standard_normal(eps.size)
        wp = _solve(ctx, eps + h * d, vectors=False)["freq"][0]
        wm = _solve(ctx, eps - h * d, vectors=False)["freq"][0]
        fd = (wp - wm) / (2 * h)
        ad = G @ d
        assert np.max(np.abs(fd - ad) / np.abs(ad)) < 1e-4, (fd, ad)


def test_autograd_matches_adjoint(setup):
    from fame_b200.autograd import band_frequencies
    _, ctx, eps, _ = setup
    e = torch.tensor(eps, dtype=torch.float64, requires_grad=True)
    w = band_frequencies(ctx, e, K, **TOLS)
    v = torch.from_numpy(np.random.default_rng(3).standard_normal(NWANT))
    (w * v).sum().backward()
    out = _solve(ctx, eps)
    G = ctx.adjoint(out["freq"][0], out["evec"][0])
    np.testing.assert_allclose(w.detach().numpy(), out["freq"][0], rtol=1e-12)
    assert _rel(e.grad.numpy(), v.numpy() @ G) < 1e-10


def test_device_resident_vjp_matches_host_adjoint(setup):
    """eps on the GPU, eigenvectors kept on the GPU, the gradient returned on the GPU:
    the same numbers as the host-side per-band adjoint contracted with grad_w."""
    from fame_b200.autograd import band_frequencies
    _, ctx, eps, _ = setup
    e = torch.tensor(eps, dtype=torch.float64, device="cuda", requires_grad=True)
    w = band_frequencies(ctx, e, K, **TOLS)
    v = torch.from_numpy(np.random.default_rng(4).standard_normal(NWANT)).to("cuda")
    (w * v).sum().backward()
    assert e.grad.is_cuda
    out = _solve(ctx, eps)
    G = ctx.adjoint(out["freq"][0], out["evec"][0])
    assert _rel(e.grad.cpu().numpy(), v.cpu().numpy() @ G) < 1e-10
    # the backward pass re-solves when another solve replaced the device eigenvectors
    w2 = band_frequencies(ctx, e, K, **TOLS)
    _solve(ctx, eps + 1.0, vectors=False)
    e.grad = None
    (w2 * v).sum().backward()
    assert _rel(e.grad.cpu().numpy(), v.cpu().numpy() @ G) < 1e-10


def test_degenerate_bands_at_x_point():
    """Simple cubic 32^3 with the dielectric sphere about the origin (the reference's
    material map: every edge tested at its own midpoint, so the discrete operator
    keeps the cubic symmetry) at X = (0.5, 0, 0): the 4-fold axis along x makes band
    pairs degenerate.  Equal weights on a degenerate pair give the derivative of the
    pair's sum: checked against central differences (step 1e-4) along a random
    voxel direction (all three edges of a voxel moved together, the voxel gradient's
    definition).  Unequal weights inside the pair are rejected."""
    par = load_pre("sc32")
    N = par["N"]
    ctx = fb.Context.from_par(par)
    from fixtures import edge_eps
    B = edge_eps(par)
    kx = np.array([[0.5, 0.0, 0.0]])
    p = fb.solver_params(**TOLS)
    ctx.set_eps_device(torch.from_numpy(B).to("cuda"))
    out = ctx.solve(kx, p, vectors_on_device=True)
    wn = out["freq"][0]
    rel = np.abs(np.diff(wn)) / wn[1:]
    pairs = [i for i in range(NWANT - 1) if rel[i] < 1e-8]
    assert pairs, wn
    i0 = pairs[0]
    wt = np.zeros(NWANT)
    wt[i0] = wt[i0 + 1] = 1.0
    g = ctx.adjoint_vjp(0, wn, wt).cpu().numpy()
    d = np.random.default_rng(11).standard_normal(N)
    h = 1e-4

    def pair_sum(Bx):
        ctx.set_eps(Bx)
        f = ctx.solve(kx, p)["freq"][0]
        return f[i0] + f[i0 + 1]

    dd = np.concatenate([d, d, d])
    fd = (pair_sum(B + h * dd) - pair_sum(B - h * dd)) / (2 * h)
    assert abs(fd - g @ d) < 1e-4 * abs(g @ d), (fd, g @ d)
    # one band of the pair alone has no derivative: rejected
    ctx.set_eps_device(torch.from_numpy(B).to("cuda"))
    out = ctx.solve(kx, p, vectors_on_device=True)
    wt = np.zeros(NWANT)
    wt[i0] = 1.0
    with pytest.raises(fb.FameError) as err:
        ctx.adjoint_vjp(0, out["freq"][0], wt)
    assert err.value.code == fb.ERR_BAD_INPUT and "degenerate" in str(err.value)
    ctx.close()
