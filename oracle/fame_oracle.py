"""CPU FP64 restatement of FAME-Isotropic-GPU's band-structure path (numpy).

TEST INFRASTRUCTURE ONLY.  This module is the oracle: tests/, the smoke check and
the cpu_baseline leg of bench.py may import it, to check results.  The product (the
CUDA library behind include/fame_b200.h) never imports, links or calls it.

Every function follows one reference routine and cites it (paths are relative
to the reference project root).  Vector layouts are the reference's:

* reduced vectors x (length 2*Nd) = [x1 (Nd), x2 (Nd)];
* 3-component fields (length 3N) = [comp x (N), comp y (N), comp z (N)];
* Simple lattices: frequency and space index idx = i + Nx*(j + Ny*k) (x fastest);
* General lattices: frequency index (i*Ny + j)*Nz + k (z fastest), space index
  x fastest (FAME_Main/FAME_FFT_CUDA.cu:63-160).

Parity pins (tests/test_oracle_*.py): the homogeneous-medium known answer, the
operator identities, integer maps produced by the reference's own preprocessing
(tests/golden/), and the reference's FP64 CUDA build run on a B200 (tests/golden/).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.linalg.lapack as _lapack

PI = 3.141592653589793  # the reference's `pi` macro (include/FAME_Internal_Common.h:23)

SIMPLE_LATTICES = ("simple_cubic", "primitive_orthorhombic", "primitive_tetragonal")


# --------------------------------------------------------------------------- Lambdas
@dataclasses.dataclass
class Lambdas:
    """Per-k operator data (FAME_Main/FAME_Matrix_Lambdas.cu:40-554)."""

    simple: bool
    grid: tuple
    Nd: int
    Lx: np.ndarray  # length N, frequency layout, full (index 0 kept)
    Ly: np.ndarray
    Lz: np.ndarray
    Lq_sqrt: np.ndarray  # length Nd
    Pi_Qr: np.ndarray  # (6, Nd)
    Pi_Pr: np.ndarray  # (6, Nd)
    D_k: np.ndarray | None = None  # Simple: length N
    D_kx: np.ndarray | None = None  # General: (Nx,)
    D_ky: np.ndarray | None = None  # General: (Nx, Ny)
    D_kz: np.ndarray | None = None  # General: (Nx, Ny, Nz)


def thetas(wave_vec, lattice_vec_a, simple, m=(0, 0, 0, 0), t1=(0.0, 0.0, 0.0), grid=None):
    """theta_x, theta_y(xy), theta_z(xyz) of FAME_Matrix_Lambdas (FAME_Matrix_Lambdas.cu:43-70)."""
    k = np.asarray(wave_vec, float)
    a = np.asarray(lattice_vec_a, float).reshape(3, 3)  # rows a1, a2, a3
    th_x = float(k @ a[0])
    if simple:
        return th_x, float(k @ a[1]), float(k @ a[2])
    m1, m2, m3, _ = m
    Nx, Ny, _ = grid
    if a[1, 0] > 0:
        c1 = -m1 / Nx
    elif a[1, 0] < 0:
        c1 = 1.0 - m1 / Nx
    else:  # the reference leaves c1 unset here; lattices it supports never hit it
        c1 = 0.0
    c2 = m3 / Ny
    c3 = m2 / Nx
    a2h = c1 * a[0] + a[1]
    a3h = a[2] - c2 * a2h - c3 * a[0] + np.asarray(t1, float)
    return th_x, float(k @ a2h), float(k @ a3h)


def _pi_simple(Lx, Ly, Lz):
    """Pi_Qr / Pi_Pr for Simple lattices (FAME_Matrix_Lambdas.cu:183-244), alpha=3, beta=5."""
    al, be = 3.0, 5.0
    Lq = (np.conj(Lx) * Lx + np.conj(Ly) * Ly + np.conj(Lz) * Lz).real
    t1 = be * Lz - Ly
    t2 = Lx - al * Lz
    t3 = al * Ly - be * Lx
    n2 = (np.conj(t1) * t1 + np.conj(t2) * t2 + np.conj(t3) * t3)
    n1 = n2 * Lq
    s1 = np.sqrt(n1.astype(complex))
    s2 = np.sqrt(n2.astype(complex))
    p1 = ((al * Ly - be * Lx) * np.conj(Ly) - (Lx - al * Lz) * np.conj(Lz)) / s1
    p2 = ((be * Lz - Ly) * np.conj(Lz) - (al * Ly - be * Lx) * np.conj(Lx)) / s1
    p3 = ((Lx - al * Lz) * np.conj(Lx) - (be * Lz - Ly) * np.conj(Ly)) / s1
    q1 = (be * np.conj(Lz) - np.conj(Ly)) / s2
    q2 = (np.conj(Lx) - al * np.conj(Lz)) / s2
    q3 = (al * np.conj(Ly) - be * np.conj(Lx)) / s2
    return Lq, np.stack([p1, p2, p3, q1, q2, q3])


def _pi_general(Lx, Ly, Lz):
    """Pi_Qr / Pi_Pr for General lattices (FAME_Matrix_Lambdas.cu:438-489)."""
    Lq = (np.conj(Lx) * Lx + np.conj(Ly) * Ly + np.conj(Lz) * Lz).real
    Ls = Lx + Ly + Lz
    Lp = np.conj(Ls) * Ls
    n1 = np.sqrt((3 * Lq * Lq - Lq * Lp).astype(complex))
    n2 = np.sqrt((3 * Lq - Lp).astype(complex))
    p1 = (Lq - Lx * np.conj(Ls)) / n1
    p2 = (Lq - Ly * np.conj(Ls)) / n1
    p3 = (Lq - Lz * np.conj(Ls)) / n1
    q1 = (np.conj(Lz) - np.conj(Ly)) / n2
    q2 = (np.conj(Lx) - np.conj(Lz)) / n2
    q3 = (np.conj(Ly) - np.conj(Lx)) / n2
    return Lq, np.stack([p1, p2, p3, q1, q2, q3])


def _finish(simple, grid, Lx, Ly, Lz, wave_vec, gamma_tol, **d):
    N = Lx.size
    Nd = N - 1 if np.linalg.norm(wave_vec) < gamma_tol else N
    s = N - Nd
    Lq, P = (_pi_simple if simple else _pi_general)(Lx[s:], Ly[s:], Lz[s:])
    Pr = np.concatenate([-np.conj(P[3:]), np.conj(P[:3])])
    return Lambdas(simple, tuple(grid), Nd, Lx, Ly, Lz, np.sqrt(Lq), P, Pr, **d)


def lambdas_simple(wave_vec, grid, mesh_len, lattice_vec_a):
    """Construct_Lambdas_Simple (FAME_Matrix_Lambdas.cu:77-286)."""
    Nx, Ny, Nz = grid
    tx, ty, tz = thetas(wave_vec, lattice_vec_a, True)
    i2pi = 2j * PI
    mx, my, mz = np.arange(Nx), np.arange(Ny), np.arange(Nz)
    L1 = (np.exp(i2pi * (mx + tx) / Nx) - 1) / mesh_len[0]
    L2 = (np.exp(i2pi * (my + ty) / Ny) - 1) / mesh_len[1]
    L3 = (np.exp(i2pi * (mz + tz) / Nz) - 1) / mesh_len[2]
    shape = (Nz, Ny, Nx)
    Lx = np.broadcast_to(L1[None, None, :], shape).ravel()
    Ly = np.broadcast_to(L2[None, :, None], shape).ravel()
    Lz = np.broadcast_to(L3[:, None, None], shape).ravel()
    Dx = np.exp(tx * i2pi * mx / Nx)
    Dy = np.exp(ty * i2pi * my / Ny)
    Dz = np.exp(tz * i2pi * mz / Nz)
    D_k = (Dz[:, None, None] * Dy[None, :, None] * Dx[None, None, :]).ravel()
    return _finish(True, grid, Lx, Ly, Lz, wave_vec, 1e-4, D_k=D_k)


def lambdas_general(wave_vec, grid, mesh_len, lattice_vec_a, m, t1):
    """Construct_Lambdas_General (FAME_Matrix_Lambdas.cu:288-554)."""
    Nx, Ny, Nz = grid
    m1, m2, m3, _ = m
    tx, txy, txyz = thetas(wave_vec, lattice_vec_a, False, m, t1, grid)
    i2pi = 2j * PI
    mx, my, mz = np.arange(Nx), np.arange(Ny), np.arange(Nz)
    L1 = (np.exp(i2pi * (mx + tx) / Nx) - 1) / mesh_len[0]
    mxy = (-(m1 / Nx) * mx)[:, None] + my[None, :]  # (Nx, Ny)
    L2 = (np.exp(i2pi * (mxy + txy) / Ny) - 1) / mesh_len[1]
    c1 = (m1 * m3) / (Ny * Nx) - (m2 / Nx)
    c2 = -(m3 / Ny)
    mxyz = (c1 * mx)[:, None, None] + (c2 * my)[None, :, None] + mz[None, None, :]
    L3 = (np.exp(i2pi * (mxyz + txyz) / Nz) - 1) / mesh_len[2]
    shape = (Nx, Ny, Nz)
    Lx = np.broadcast_to(L1[:, None, None], shape).ravel()
    Ly = np.broadcast_to(L2[:, :, None], shape).ravel()
    Lz = L3.ravel()
    D_kx = np.exp(tx * i2pi * mx / Nx)
    phi_jx = i2pi * (txy + mx * (-m1 / Nx)) / Ny  # (Nx,)
    D_ky = np.exp(phi_jx[:, None] * my[None, :])
    phi_k = i2pi * (txyz + my[None, :] * (-m3 / Ny)
                    + mx[:, None] * ((m1 * m3) / (Nx * Ny) - m2 / Nx)) / Nz
    D_kz = np.exp(phi_k[:, :, None] * mz[None, None, :])
    return _finish(False, grid, Lx, Ly, Lz, wave_vec, 1e-3, D_kx=D_kx, D_ky=D_ky, D_kz=D_kz)


def lambdas(wave_vec, par):
    """FAME_Matrix_Lambdas dispatch (FAME_Matrix_Lambdas.cu:40-76)."""
    if par["simple"]:
        return lambdas_simple(wave_vec, par["grid"], par["mesh_len"], par["lattice_vec_a"])
    return lambdas_general(wave_vec, par["grid"], par["mesh_len"], par["lattice_vec_a"],
                           par["m"], par["t1"])


# ------------------------------------------------------------------ transforms
def _T_general(p, L: Lambdas):
    """spMV_fastT_gpu flag=+1 on one component (FAME_FFT_CUDA.cu:104-125)."""
    Nx, Ny, Nz = L.grid
    a = p.reshape(Nx, Ny, Nz)
    a = np.fft.ifft(a, axis=2) * Nz
    a = a * L.D_kz
    a = np.fft.ifft(a, axis=1) * Ny
    a = a * L.D_ky[:, :, None]
    a = np.fft.ifft(a, axis=0) * Nx
    a = a * L.D_kx[:, None, None] / (Nx * Ny * Nz)
    return np.ascontiguousarray(a.transpose(2, 1, 0)).ravel()


def _Ts_general(v, L: Lambdas):
    """spMV_fastT_gpu flag=-1 on one component (FAME_FFT_CUDA.cu:128-150)."""
    Nx, Ny, Nz = L.grid
    a = v.reshape(Nz, Ny, Nx).transpose(2, 1, 0)
    a = a * np.conj(L.D_kx)[:, None, None]
    a = np.fft.fft(a, axis=0)
    a = a * np.conj(L.D_ky)[:, :, None]
    a = np.fft.fft(a, axis=1)
    a = a * np.conj(L.D_kz)
    a = np.fft.fft(a, axis=2)
    return np.ascontiguousarray(a).ravel()


def _inv3d(t, L: Lambdas):
    Nx, Ny, Nz = L.grid
    if L.simple:  # IFFT_CUDA (FAME_FFT_CUDA.cu:38-60): unnormalised inverse, x1/N, D_k
        return L.D_k * np.fft.ifftn(t.reshape(Nz, Ny, Nx)).ravel()
    return _T_general(t, L)


def _fwd3d(v, L: Lambdas):
    Nx, Ny, Nz = L.grid
    if L.simple:  # FFT_CUDA (FAME_FFT_CUDA.cu:18-36): D_ks then unnormalised forward
        return np.fft.fftn((np.conj(L.D_k) * v).reshape(Nz, Ny, Nx)).ravel()
    return _Ts_general(v, L)


def _mix(x, P, L: Lambdas):
    """vp_add_vp into a zeroed 3N buffer at offset N-Nd (…_Qr.cu:29-35, …_Pr.cu:162-175)."""
    N, Nd = L.Lx.size, L.Nd
    t = np.zeros((3, N), complex)
    for c in range(3):
        t[c, N - Nd:] = P[c] * x[:Nd] + P[3 + c] * x[Nd:2 * Nd]
    return t


def Qr(x, L: Lambdas):
    """FAME_Matrix_Vector_Production_Qr (FAME_Matrix_Vector_Production_Qr.cu:8-78)."""
    t = _mix(x, L.Pi_Qr, L)
    return np.concatenate([_inv3d(t[c], L) for c in range(3)])


def Pr(x, L: Lambdas):
    """FAME_Matrix_Vector_Production_Pr (FAME_Matrix_Vector_Production_Pr.cu:11-104)."""
    t = _mix(x, L.Pi_Pr, L)
    return np.concatenate([_inv3d(t[c], L) for c in range(3)])


def _unmix(t, P, L: Lambdas):
    """vp_add_vp_add_vp with Pi_Qrs = conj(Pi_Qr) reordered (…_Qrs.cu:61-76)."""
    N, Nd = L.Lx.size, L.Nd
    tt = [t[c][N - Nd:] for c in range(3)]
    o1 = sum(np.conj(P[c]) * tt[c] for c in range(3))
    o2 = sum(np.conj(P[3 + c]) * tt[c] for c in range(3))
    return np.concatenate([o1, o2])


def Qrs(v, L: Lambdas):
    """FAME_Matrix_Vector_Production_Qrs (FAME_Matrix_Vector_Production_Qrs.cu:7-58)."""
    N = L.Lx.size
    t = [_fwd3d(v[c * N:(c + 1) * N], L) for c in range(3)]
    return _unmix(t, L.Pi_Qr, L)


def Prs(v, L: Lambdas):
    """FAME_Matrix_Vector_Production_Prs (FAME_Matrix_Vector_Production_Prs.cu:9-58)."""
    N = L.Lx.size
    t = [_fwd3d(v[c * N:(c + 1) * N], L) for c in range(3)]
    return _unmix(t, L.Pi_Pr, L)


def QBQ(x, L: Lambdas, invB):
    """FAME_Matrix_Vector_Production_Isotropic_QBQ (…_QBQ.cu:8-67)."""
    return Qrs(Qr(x, L) * invB, L)


# ------------------------------------------------------------------ CG / invAr
def cg(apply, rhs, tol, maxit):
    """CG with x0 = 0 and an absolute tolerance on ||r|| (FAME_Main/CG.cu:5-88).

    Returns (x, k) where k is the reference's iteration counter (it starts at 1,
    so a solve doing m products returns m + 1)."""
    x = np.zeros_like(rhs)
    r = rhs.copy()
    r1 = np.vdot(r, r).real
    p = None
    r0 = None
    k = 1
    while r1 > tol * tol and k <= maxit:
        if k > 1:
            p = r + (r1 / r0) * p
        else:
            p = r.copy()
        Ap = apply(p)
        dot = np.vdot(p, Ap)
        a = r1 / dot  # = r1*conj(dot)/|dot|^2, CG.cu:60-63
        x = x + a * p
        r = r - a * Ap
        r0 = r1
        r1 = np.vdot(r, r).real
        k += 1
    return x, k


def invAr(x, L: Lambdas, invB, tol, maxit, counters=None):
    """FAME_Matrix_Vector_Production_Isotropic_invAr (…_invAr.cu:8-48)."""
    s = np.concatenate([L.Lq_sqrt, L.Lq_sqrt])
    y, k = cg(lambda p: QBQ(p, L, invB), x / s, tol, maxit)
    if counters is not None:
        counters["ls_iter"] += k
        counters["es_iter"] += 1
    return y / s


# ------------------------------------------------------------------ Lanczos
def given_rotation(a, b):
    """given_rotation (FAME_Main/Lanczos_LockPurge_gpu.cu:245-265); returns c, s, r."""
    if abs(a) > abs(b):
        t = b / a
        u = abs(a) / a * math.sqrt(1 + t * t)
        c = 1.0 / u
        s = c * t
        r = a * u
        s = -s
    else:
        t = a / b
        u = abs(b) / b * math.sqrt(1 + t * t)
        s = 1.0 / u
        c = s * t
        r = b * u
        s = -s
    return c, s, r


def gvqrrq(T0, T1, shift, n):
    """One shifted QR step on the leading n x n tridiagonal, in place
    (GVqrrq_g, FAME_Main/Lanczos_LockPurge_gpu.cu:95-190).  Returns c, s (n-1)."""
    c = np.zeros(max(n - 1, 0))
    s = np.zeros(max(n - 1, 0))
    T2 = np.zeros(max(n - 2, 1))
    T3 = T1[:n - 1].copy()
    for i in range(n):
        T0[i] -= shift
    for i in range(n - 1):
        a, b = T0[i], T1[i]
        c[i], s[i], r = given_rotation(a, b)
        T0[i] = r
        T1[i] = 0.0
        a, b = T3[i], T0[i + 1]
        T3[i] = c[i] * a - s[i] * b
        T0[i + 1] = s[i] * a + c[i] * b
        if i < n - 2:
            T2[i] = -s[i] * T3[i + 1]
            T3[i + 1] = c[i] * T3[i + 1]
    R0, R1, R2, R3 = T0[0], T3[0], T1[0], T0[1]
    T0[0] = c[0] * R0 - s[0] * R1
    T3[0] = s[0] * R0 + c[0] * R1
    T1[0] = c[0] * R2 - s[0] * R3
    T0[1] = s[0] * R2 + c[0] * R3
    for i in range(1, n - 1):
        R = (T3[i - 1], T2[i - 1], T0[i], T3[i], T1[i], T0[i + 1])
        T3[i - 1] = c[i] * R[0] - s[i] * R[1]
        T2[i - 1] = s[i] * R[0] + c[i] * R[1]
        T0[i] = c[i] * R[2] - s[i] * R[3]
        T3[i] = s[i] * R[2] + c[i] * R[3]
        T1[i] = c[i] * R[4] - s[i] * R[5]
        T0[i + 1] = s[i] * R[4] + c[i] * R[5]
    for i in range(n - 1):
        T1[i] = (T1[i] + T3[i]) / 2.0
    for i in range(n):
        T0[i] += shift
    return c, s


def _zdrot(x, y, c, s):
    """cublasZdrot: x' = c x + s y, y' = -s x + c y (real c, s)."""
    return c * x + s * y, -s * x + c * y


def lock_purge(U, T0, T1, LT0, nwant, nstep):
    """Lanczos_LockPurge_gpu (FAME_Main/Lanczos_LockPurge_gpu.cu:7-48), in place.
    U has nstep+1 columns (U[:, j])."""
    for j in range(nstep - nwant):
        n = nstep - j
        c, s = gvqrrq(T0, T1, LT0[nwant + j], n)
        for jj in range(n - 1):
            U[:, jj + 1], U[:, jj] = _zdrot(U[:, jj + 1], U[:, jj], c[jj], s[jj])
        jj = n - 1
        s[jj - 1] *= T1[jj]
        U[:, jj + 1], U[:, jj] = _zdrot(U[:, jj + 1], U[:, jj], T1[jj - 1], s[jj - 1])
        T1[jj - 1] = np.linalg.norm(U[:, jj])
        U[:, jj] *= 1.0 / T1[jj - 1]
        T0[jj] = 0.0
        T1[jj] = 0.0
        U[:, jj + 1] = 0.0


def lanczos_decomp(U, T0, T1, is_init, op, nwant, nstep):
    """Lanczos_decomp_gpu (FAME_Main/Lanczos_decomp_gpu.cu:7-91), in place."""
    M = U.shape[0]
    if not is_init:
        U[:, 0] = 0.0
        U[M - 1, 0] = 1.0  # e_M, Lanczos_init_kernel (:93-107)
        U[:, 1] = op(U[:, 0])
        T0[0] = np.vdot(U[:, 1], U[:, 0]).real
        U[:, 1] -= T0[0] * U[:, 0]
        T1[0] = np.linalg.norm(U[:, 1])
        U[:, 1] *= 1.0 / T1[0]
        start = 1
    else:
        start = nwant
    for j in range(start, nstep):
        w = op(U[:, j])
        T0[j] = np.vdot(w, U[:, j]).real
        w = w - T0[j] * U[:, j]
        w = w - T1[j - 1] * U[:, j - 1]
        T1[j] = np.linalg.norm(w)
        w = w * (1.0 / T1[j])
        for i in range(j + 1):  # one MGS pass, no renormalisation (:80-87)
            w = w - np.vdot(U[:, i], w) * U[:, i]
        U[:, j + 1] = w


def zpteqr(d, e):
    """LAPACKE_zpteqr(COL_MAJOR, 'I', ...) as called at Lanczos_Isotropic.cu:53
    (LAPACK 3.8.0, a third-party dependency; here the same routine from scipy's
    LAPACK).  Returns eigenvalues (descending) and Z (column-major semantics: Z[:, i])."""
    n = d.size
    dd, ee, z, info = _lapack.zpteqr(d.copy(), e.copy(), np.zeros((n, n), complex), compute_z=2)
    if info != 0:
        raise RuntimeError(f"zpteqr info={info}")
    return dd, z


@dataclasses.dataclass
class LanczosResult:
    freq: np.ndarray
    ev: np.ndarray  # (2Nd, nwant) Ritz vectors
    restarts: int
    converged: bool
    theta: np.ndarray  # Ritz values of A_r^{-1}, descending


def lanczos(op, M, nwant, nstep, tol, maxit):
    """Lanczos_Isotropic (FAME_Main/Lanczos_Isotropic.cu:7-96)."""
    U = np.zeros((M, nstep + 1), complex)
    T0 = np.zeros(nstep)
    T1 = np.zeros(nstep)
    lanczos_decomp(U, T0, T1, False, op, nwant, nstep)
    it = 1
    conv_all = False
    LT0 = None
    z = None
    while it <= maxit:
        LT0, z = zpteqr(T0.copy(), T1[:nstep - 1].copy())
        conv = 0
        for i in range(nwant):
            res = T1[nstep - 1] * abs(z[nstep - 1, i])
            if res < tol:
                conv += 1
            else:
                break
        if conv == nwant:
            conv_all = True
            break
        lock_purge(U, T0, T1, LT0, nwant, nstep)
        lanczos_decomp(U, T0, T1, True, op, nwant, nstep)
        it += 1
    freq = np.sqrt(1.0 / LT0[:nwant])
    ev = U[:, :nstep] @ z[:, :nwant]
    return LanczosResult(freq, ev, it, conv_all, LT0)


def restore(ev, L: Lambdas, invB):
    """Eigen_Restoration_Isotropic (FAME_Fast_Algorithms_Isotropic.cu:90-125):
    E = B^{-1} Q_r (Sigma ev), then scaled BY its norm (the reference multiplies by
    the norm, :119-121)."""
    s = np.concatenate([L.Lq_sqrt, L.Lq_sqrt])
    out = []
    for i in range(ev.shape[1]):
        e = Qr(ev[:, i] * s, L) * invB
        out.append(e * np.linalg.norm(e))
    return np.stack(out, axis=1)


def gamma_patch(freq, E, N):
    """Gamma-point patch of FAME_Fast_Algorithms_Isotropic (:61-79)."""
    f = freq.copy()
    E = E.copy()
    nw = f.size
    f[2:] = freq[:nw - 2]
    E[:, 2:] = E[:, :nw - 2].copy()
    f[:2] = 0.0
    E[:, :2] = 1.0 / math.sqrt(3 * N)
    return f, E


@dataclasses.dataclass
class SolveResult:
    freq: np.ndarray
    E: np.ndarray
    Nd: int
    ls_iter: int
    es_iter: int
    restarts: int
    converged: bool


def solve_k(wave_vec, par, B, es, ls):
    """FAME_Fast_Algorithms_Isotropic for one k (FAME_Fast_Algorithms_Isotropic.cu:20-86).

    es = dict(nwant, nstep, tol, maxit); ls = dict(tol, maxit); B: 3N edge eps."""
    L = lambdas(wave_vec, par)
    invB = 1.0 / B
    cnt = {"ls_iter": 0, "es_iter": 0}
    op = lambda u: invAr(u, L, invB, ls["tol"], ls["maxit"], cnt)
    res = lanczos(op, 2 * L.Nd, es["nwant"], es["nstep"], es["tol"], es["maxit"])
    E = restore(res.ev, L, invB)
    N = L.Lx.size
    f = res.freq
    if L.Nd == N - 1:
        f, E = gamma_patch(f, E, N)
    return SolveResult(f, E, L.Nd, cnt["ls_iter"], cnt["es_iter"], res.restarts, res.converged)


# ------------------------------------------------------------------ material / B
def hellmann_feynman_voxel_gradient(E, freq, B, N):
    """d w_i / d eps_v for C^H C E = w^2 B E with one permittivity per voxel on its
    three edges: -(w_i / 2) sum_c |E_i,c,v|^2 / (E_i^H B E_i).  E: (nwant, 3N),
    freq: (nwant,), B: (3N,).  The reference has no adjoint; this is the textbook
    first-order perturbation of a generalized Hermitian eigenvalue, used to check
    the adjoint kernel against the reference's own eigenvectors."""
    E = np.asarray(E).reshape(len(freq), 3 * N)
    a2 = np.abs(E) ** 2
    den = a2 @ B
    g = a2[:, :N] + a2[:, N:2 * N] + a2[:, 2 * N:]
    w = np.asarray(freq, dtype=float)
    out = -(w / 2.0)[:, None] * g / den[:, None]
    out[w <= 0] = 0.0
    return out


def matrix_B(binout, material_num, eps_in, eps_out, N):
    """FAME_Matrix_B_Isotropic (FAME_Main/FAME_Matrix_B_Isotropic.cu:4-74): the last
    matching material wins."""
    B = np.full(3 * N, float(eps_out))
    b = np.asarray(binout).reshape(3, material_num, N)
    for c in range(3):
        for j in range(material_num):
            B[c * N:(c + 1) * N][b[c, j] == 1] = eps_in[j]
    return B


# ------------------------------------------------------------------ sparse curl
def _k1d(n, h, theta):
    """spMTX_FDM_1d_quasiperiodic (FAME_Matrix_Curl.cpp:378-397) as a dense-free
    operator: (K x)[i] = (x[i+1]-x[i])/h, wrap with e^{theta}."""
    def f(x, axis):
        xp = np.roll(x, -1, axis=axis)
        idx = [slice(None)] * x.ndim
        idx[axis] = n - 1
        xp[tuple(idx)] *= np.exp(theta)
        return (xp - x) / h
    return f


def curl_simple_apply(E, wave_vec, par):
    """C E for Simple lattices, C = [[0,-C3,C2],[C3,0,-C1],[-C2,C1,0]] with
    C1 = I_z (x) I_y (x) K_x etc. (FAME_Matrix_Curl.cpp:90-219)."""
    Nx, Ny, Nz = par["grid"]
    h = par["mesh_len"]
    a = np.asarray(par["lattice_vec_a"], float).reshape(3, 3)
    k = np.asarray(wave_vec, float)
    th = [2j * PI * float(a[i] @ k) for i in range(3)]
    N = Nx * Ny * Nz
    e = [E[c * N:(c + 1) * N].reshape(Nz, Ny, Nx) for c in range(3)]
    d1 = _k1d(Nx, h[0], th[0])
    d2 = _k1d(Ny, h[1], th[1])
    d3 = _k1d(Nz, h[2], th[2])
    C1 = lambda u: d1(u, 2)
    C2 = lambda u: d2(u, 1)
    C3 = lambda u: d3(u, 0)
    out = [-C3(e[1]) + C2(e[2]), C3(e[0]) - C1(e[2]), -C2(e[0]) + C1(e[1])]
    return np.concatenate([o.ravel() for o in out])


def curl_simple_apply_H(F, wave_vec, par):
    """C^H F for Simple lattices (adjoint of curl_simple_apply)."""
    Nx, Ny, Nz = par["grid"]
    h = par["mesh_len"]
    a = np.asarray(par["lattice_vec_a"], float).reshape(3, 3)
    k = np.asarray(wave_vec, float)
    th = [2j * PI * float(a[i] @ k) for i in range(3)]
    N = Nx * Ny * Nz

    def kH(n, hh, theta, axis):
        def f(y):
            # K^H y: (K^H y)[i] = (y[i-1] - y[i])/h with y[-1] -> conj(e^theta) y[n-1]
            ym = np.roll(y, 1, axis=axis)
            idx = [slice(None)] * y.ndim
            idx[axis] = 0
            ym[tuple(idx)] *= np.conj(np.exp(theta))
            return (ym - y) / hh
        return f

    f = [F[c * N:(c + 1) * N].reshape(Nz, Ny, Nx) for c in range(3)]
    C1H = kH(Nx, h[0], th[0], 2)
    C2H = kH(Ny, h[1], th[1], 1)
    C3H = kH(Nz, h[2], th[2], 0)
    # C^H = [[0, C3^H, -C2^H], [-C3^H, 0, C1^H], [C2^H, -C1^H, 0]]
    out = [C3H(f[1]) - C2H(f[2]), -C3H(f[0]) + C1H(f[2]), C2H(f[0]) - C1H(f[1])]
    return np.concatenate([o.ravel() for o in out])


def relative_residual_simple(E, omega, wave_vec, par, B):
    """||C^H C E - w^2 B E|| / (w^2 ||B E||) with the independent sparse curl
    (Check_Residual's quantity, FAME_Main_Code.cu:383-421, made relative)."""
    CE = curl_simple_apply(E, wave_vec, par)
    lhs = curl_simple_apply_H(CE, wave_vec, par)
    BE = B * E
    w2 = omega * omega
    return np.linalg.norm(lhs - w2 * BE) / (w2 * np.linalg.norm(BE))


# ------------------------------------------------------------------ material locate
def _grid_point(i, j, k, mesh_len, comp):
    sh = [0.0, 0.0, 0.0]
    sh[comp] = 0.5
    return ((i + sh[0]) * mesh_len[0], (j + sh[1]) * mesh_len[1], (k + sh[2]) * mesh_len[2])


def material_locate(par, material):
    """FAME_Material_Locate_Index (FAME_Preprocessing/FAME_Material_Locate_Index.cpp:6-113,
    FAME_Material_Handle.cpp:4-87, FAME_Matrix_Grid.cpp:4-53), vectorised over the
    grid with the same floating-point operation order.  Returns Binout (int32,
    3 * material_num * N)."""
    Nx, Ny, Nz = par["grid"]
    N = Nx * Ny * Nz
    h = par["mesh_len"]
    Om = np.asarray(par["Omega"], float)
    A = np.asarray(par["lattice_vec_a"], float)
    perm = list(par["Permutation"])
    # lattice_vec_a_orig_P = Omega' * lattice_vec_a (column i of the product)
    AP = np.zeros(9)
    cnt = 0
    for i in range(3):
        AP[i] = Om[cnt] * A[0] + Om[cnt + 1] * A[1] + Om[cnt + 2] * A[2]
        AP[i + 3] = Om[cnt] * A[3] + Om[cnt + 1] * A[4] + Om[cnt + 2] * A[5]
        AP[i + 6] = Om[cnt] * A[6] + Om[cnt + 1] * A[7] + Om[cnt + 2] * A[8]
        cnt += 3
    invAP = _inv3(AP)
    if perm == [2, 3, 1]:
        invP = [3, 1, 2]
    elif perm == [3, 1, 2]:
        invP = [2, 3, 1]
    else:
        invP = perm
    Aorig = np.concatenate([AP[(invP[q] - 1) * 3:(invP[q] - 1) * 3 + 3] for q in range(3)])
    nm = material["material_num"]
    out = np.zeros((3, nm, N), np.int32)
    kk, jj, ii = np.meshgrid(np.arange(Nz), np.arange(Ny), np.arange(Nx), indexing="ij")
    for comp in range(3):
        sh = [0.0, 0.0, 0.0]
        sh[comp] = 0.5
        p0 = ((ii + sh[0]) * h[0]).ravel()
        p1 = ((jj + sh[1]) * h[1]).ravel()
        p2 = ((kk + sh[2]) * h[2]).ravel()
        o0 = p0 * Om[0] + p1 * Om[1] + p2 * Om[2]
        o1 = p0 * Om[3] + p1 * Om[4] + p2 * Om[5]
        o2 = p0 * Om[6] + p1 * Om[7] + p2 * Om[8]
        c0 = o0 * invAP[0] + o1 * invAP[3] + o2 * invAP[6]
        c1 = o0 * invAP[1] + o1 * invAP[4] + o2 * invAP[7]
        c2 = o0 * invAP[2] + o1 * invAP[5] + o2 * invAP[8]
        s1, s2, s3 = np.floor(c0), np.floor(c1), np.floor(c2)
        q0 = o0 - (s1 * AP[0] + s2 * AP[3] + s3 * AP[6])
        q1 = o1 - (s1 * AP[1] + s2 * AP[4] + s3 * AP[7])
        q2 = o2 - (s1 * AP[2] + s2 * AP[5] + s3 * AP[8])
        assigned = np.zeros(N, bool)
        for kind in range(nm):
            hit = _sphere_hits(q0, q1, q2, Aorig, material, kind) | \
                _cylinder_hits(q0, q1, q2, Aorig, material, kind)
            new = hit & ~assigned
            out[comp, kind, new] = 1
            assigned |= hit
    return out.ravel()


def _sphere_hits(px, py, pz, A, mat, kind):
    start = sum(mat["sphere_num"][:kind])
    hit = np.zeros(px.shape, bool)
    C = mat["sphere_centers"]
    R = mat["sphere_radius"]
    for i in range(start, start + mat["sphere_num"][kind]):
        for sx in (-1, 0, 1):
            for sy in (-1, 0, 1):
                for sz in (-1, 0, 1):
                    u, v, w = C[3 * i] + sx, C[3 * i + 1] + sy, C[3 * i + 2] + sz
                    cx = u * A[0] + v * A[3] + w * A[6]
                    cy = u * A[1] + v * A[4] + w * A[7]
                    cz = u * A[2] + v * A[5] + w * A[8]
                    d = (cx - px) ** 2 + (cy - py) ** 2 + (cz - pz) ** 2
                    hit |= d <= R[i] ** 2
    return hit


def _cylinder_hits(px, py, pz, A, mat, kind):
    start = sum(mat["cylinder_num"][:kind])
    hit = np.zeros(px.shape, bool)
    T = mat["cylinder_top_centers"]
    Bc = mat["cylinder_bot_centers"]
    R = mat["cylinder_radius"]
    for i in range(start, start + mat["cylinder_num"][kind]):
        for sx in (-1, 0, 1):
            for sy in (-1, 0, 1):
                for sz in (-1, 0, 1):
                    u, v, w = T[3 * i] + sx, T[3 * i + 1] + sy, T[3 * i + 2] + sz
                    tx = u * A[0] + v * A[3] + w * A[6]
                    ty = u * A[1] + v * A[4] + w * A[7]
                    tz = u * A[2] + v * A[5] + w * A[8]
                    u, v, w = Bc[3 * i] + sx, Bc[3 * i + 1] + sy, Bc[3 * i + 2] + sz
                    bx = u * A[0] + v * A[3] + w * A[6]
                    by = u * A[1] + v * A[4] + w * A[7]
                    bz = u * A[2] + v * A[5] + w * A[8]
                    den = (bx - tx) ** 2 + (by - ty) ** 2 + (bz - tz) ** 2
                    t = ((px - tx) * (bx - tx) + (py - ty) * (by - ty) + (pz - tz) * (bz - tz)) / den
                    inside = (0.0 <= t) & (t <= 1.0)
                    d = (tx + t * (bx - tx) - px) ** 2 + (ty + t * (by - ty) - py) ** 2 \
                        + (tz + t * (bz - tz) - pz) ** 2
                    hit |= inside & (d <= R[i] ** 2)
    return hit


def _inv3(A):
    """inv3 (FAME_Tools/inv3.cpp:8-23): adjugate/determinant inverse of a
    column-major 3x3, with the reference's operation order (Binout must be
    bit-exact, so the floor() inputs must round identically)."""
    A = [float(v) for v in A]
    det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[3] * (A[1] * A[8] - A[7] * A[2]) \
        + A[6] * (A[1] * A[5] - A[4] * A[2])
    inv = 1 / det
    return np.array([
        (A[4] * A[8] - A[5] * A[7]) * inv,
        -(A[1] * A[8] - A[2] * A[7]) * inv,
        (A[1] * A[5] - A[2] * A[4]) * inv,
        -(A[3] * A[8] - A[6] * A[5]) * inv,
        (A[0] * A[8] - A[6] * A[2]) * inv,
        -(A[0] * A[5] - A[2] * A[3]) * inv,
        (A[3] * A[7] - A[6] * A[4]) * inv,
        -(A[0] * A[7] - A[1] * A[6]) * inv,
        (A[0] * A[4] - A[1] * A[3]) * inv,
    ])
