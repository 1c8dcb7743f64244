"""Band frequencies as a differentiable function of the voxel permittivity.

`BandFrequencies` is a torch.autograd.Function around the C ABI: the forward pass
solves one k-point (fame_solve_kpoints, eigenvectors kept), the backward pass runs
the Hellmann-Feynman adjoint kernel (fame_adjoint).  For C^H C E = w^2 B E with a
diagonal B, d(w^2)/dB_e = -w^2 |E_e|^2 / (E^H B E); one permittivity per voxel sets
the x, y and z edges of that voxel (B_x = B_y = B_z = eps, edge index i + Nx (j + Ny k)),
so dw/d eps_v sums the three edges.  Non-degenerate bands only; bands pinned to
w = 0 at the Gamma point get zero gradient.  The reference has no adjoint.

    ctx = fame_b200.Context(grid, mesh_len, lattice_vec_a, simple)
    eps = torch.tensor(eps_voxels, dtype=torch.float64, requires_grad=True)
    w = band_frequencies(ctx, eps, k, nwant=8)   # (nwant,) float64
    w.sum().backward()                          # eps.grad: (N,)
"""
from __future__ import annotations

import numpy as np
import torch

from . import FP64, solver_params


def edges_from_voxels(eps_voxel: np.ndarray) -> np.ndarray:
    """B (3N) with one permittivity per voxel on its x, y and z edges."""
    e = np.ascontiguousarray(eps_voxel, dtype=np.float64).reshape(-1)
    return np.concatenate([e, e, e])


class BandFrequencies(torch.autograd.Function):
    """w(eps) for one k-point; eps is the voxel permittivity (N,), float64."""

    @staticmethod
    def forward(fctx, eps, ctx, k, params):
        B = edges_from_voxels(eps.detach().cpu().numpy())
        ctx.set_eps(B)
        p = params
        p.want_vectors = 1
        out = ctx.solve(np.asarray(k, dtype=np.float64).reshape(1, 3), p)
        freq = out["freq"][0].copy()
        fctx.fame = (ctx, B, freq, out["evec"][0])
        fctx.device = eps.device
        return torch.from_numpy(freq).to(eps.device)

    @staticmethod
    def backward(fctx, grad_w):
        ctx, B, freq, evec = fctx.fame
        ctx.set_eps(B)  # the adjoint reads the forward pass's B
        G = ctx.adjoint(freq, evec)  # (nwant, N): d w_i / d eps_v
        g = grad_w.detach().cpu().numpy().astype(np.float64) @ G
        return torch.from_numpy(g).to(fctx.device), None, None, None


def band_frequencies(ctx, eps, k, nwant=8, precision=FP64, **solver_kw):
    """Differentiable band frequencies at wave vector k (the reference's convention:
    Cartesian, without the 2*pi factor).  solver_kw go to solver_params."""
    kw = dict(nwant=nwant, nstep=40, es_tol=1e-12, ls_tol=1e-12, es_maxit=100, ls_maxit=1000,
              precision=precision)
    kw.update(solver_kw)
    return BandFrequencies.apply(eps, ctx, k, solver_params(**kw))
