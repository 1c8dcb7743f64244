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
