"""Band frequencies as a differentiable function of the voxel permittivity.

`BandFrequencies` is a torch.autograd.Function around the C ABI.  The forward pass
uploads the permittivity from its device tensor (fame_set_eps_device) and solves one
k-point with the eigenvectors kept on the GPU (fame_solve_kpoints, evec_out NULL).
The backward pass runs the Hellmann-Feynman adjoint on the device and returns the
vector-Jacobian product sum_i grad_w_i dw_i/deps_v as a device tensor
(fame_adjoint_vjp): nothing of size N crosses to the host.  For C^H C E = w^2 B E
with a diagonal B, d(w^2)/dB_e = -w^2 |E_e|^2 / (E^H B E); one permittivity per
voxel sets the x, y and z edges of that voxel (B_x = B_y = B_z = eps, edge index
i + Nx (j + Ny k)), so dw/d eps_v sums the three edges.  Bands pinned to w = 0 at the
Gamma point get zero gradient.  Degenerate bands (relative gap <= rel_gap) must
carry equal weights in grad_w: the derivative of one band of a degenerate group is
not defined, that of the group's sum is.  The reference has no adjoint.

    ctx = fame_b200.Context(grid, mesh_len, lattice_vec_a, simple)
    eps = torch.tensor(eps_voxels, dtype=torch.float64, device="cuda", requires_grad=True)
    w = band_frequencies(ctx, eps, k, nwant=8)   # (nwant,) float64
    w.sum().backward()                          # eps.grad: (N,) on the GPU
"""
from __future__ import annotations

import numpy as np
import torch

from . import FP64, OK, FameError, solver_params


def edges_from_voxels(eps_voxel: np.ndarray) -> np.ndarray:
    """B (3N) with one permittivity per voxel on its x, y and z edges."""
    e = np.ascontiguousarray(eps_voxel, dtype=np.float64).reshape(-1)
    return np.concatenate([e, e, e])


def _forward(ctx, B, k, params):
    ctx.set_eps_device(B)
    out = ctx.solve(np.asarray(k, dtype=np.float64).reshape(1, 3), params, vectors_on_device=True)
    if out["rc"] != OK:
        raise FameError(out["rc"], "band solve did not converge")
    return out["freq"][0].copy(), ctx.solves


class BandFrequencies(torch.autograd.Function):
    """w(eps) for one k-point; eps is the voxel permittivity (N,), float64."""

    @staticmethod
    def forward(fctx, eps, ctx, k, params, rel_gap):
        dev = torch.device(f"cuda:{ctx.device}")
        e = eps.detach().to(dev, torch.float64).contiguous()
        B = torch.cat([e, e, e])
        freq, serial = _forward(ctx, B, k, params)
        fctx.fame = (ctx, B, k, params, freq, serial, rel_gap)
        fctx.eps_device = eps.device
        return torch.from_numpy(freq).to(eps.device)

    @staticmethod
    def backward(fctx, grad_w):
        ctx, B, k, params, freq, serial, rel_gap = fctx.fame
        if ctx.solves != serial:
            # another solve replaced the device eigenvectors (and B): redo this one
            freq2, _ = _forward(ctx, B, k, params)
            if not np.allclose(freq2, freq, rtol=1e-10, atol=0):
                raise RuntimeError("re-solve for the adjoint changed the frequencies")
        g = ctx.adjoint_vjp(0, freq, grad_w.detach().to("cpu", torch.float64).numpy(), rel_gap)
        return g.to(fctx.eps_device), None, None, None, None


def band_frequencies(ctx, eps, k, nwant=8, precision=FP64, rel_gap=1e-6, **solver_kw):
    """Differentiable band frequencies at wave vector k (the reference's convention:
    Cartesian, without the 2*pi factor).  solver_kw go to solver_params."""
    kw = dict(nwant=nwant, nstep=40, es_tol=1e-12, ls_tol=1e-12, es_maxit=100, ls_maxit=1000,
              precision=precision)
    kw.update(solver_kw)
    return BandFrequencies.apply(eps, ctx, k, solver_params(**kw), rel_gap)
