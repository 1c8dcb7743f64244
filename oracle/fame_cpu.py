"""ctypes binding of oracle/fame_cpu.cpp (oracle/_build/libfame_cpu.so): the C++ /
OpenMP FP64 restatement of the plain method on Simple lattices.

TEST INFRASTRUCTURE ONLY: tests/ and the cpu_baseline leg of bench.py use it to
check results and as the CPU baseline.  The product never imports it."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libfame_cpu.so")
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"{LIB} not built (make -C oracle)")
        lib = C.CDLL(LIB)
        D, I = C.POINTER(C.c_double), C.POINTER(C.c_int)
        lib.fame_cpu_solve.argtypes = [I, D, D, D, D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double,
                                       C.c_int, C.c_int, D, I, I, I, I, D]
        lib.fame_cpu_solve.restype = C.c_int
        lib.fame_cpu_time.argtypes = [I, D, D, D, D, C.c_int, C.c_int, C.c_int, D, D]
        lib.fame_cpu_time.restype = C.c_int
        lib.fame_cpu_threads.restype = C.c_int
        _lib = lib
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def threads():
    return load().fame_cpu_threads()


def solve(par, B, kpoints, nwant, nstep, es_tol, es_maxit, ls_tol, ls_maxit, nthreads=0):
    """Plain FP64 solve of every k-point (Simple lattices).  Returns dict(freq,
    ls_iter, es_iter, restarts, converged, wall_s)."""
    if not par["simple"]:
        raise ValueError("the C++ restatement covers Simple lattices")
    k = _d(np.asarray(kpoints).reshape(-1, 3))
    nk = k.shape[0]
    grid = np.ascontiguousarray(par["grid"], dtype=np.int32)
    h, a, b = _d(par["mesh_len"]), _d(np.asarray(par["lattice_vec_a"]).reshape(9)), _d(B)
    freq = np.zeros((nk, nwant))
    ls, es, rs, cv = (np.zeros(nk, dtype=np.int32) for _ in range(4))
    wall = np.zeros(nk)
    rc = load().fame_cpu_solve(_p(grid, C.c_int), _p(h), _p(a), _p(b), _p(k), nk, nwant, nstep, es_tol, es_maxit,
                               ls_tol, ls_maxit, nthreads, _p(freq), _p(ls, C.c_int), _p(es, C.c_int),
                               _p(rs, C.c_int), _p(cv, C.c_int), _p(wall))
    if rc:
        raise RuntimeError("tridiagonal eigensolve failed")
    return dict(freq=freq, ls_iter=ls, es_iter=es, restarts=rs, converged=cv, wall_s=wall)


def time_blocks(par, B, k, iters=20, jstep=25, nthreads=0):
    """(seconds per CG iteration, seconds per Lanczos step at j = jstep) at k."""
    grid = np.ascontiguousarray(par["grid"], dtype=np.int32)
    h, a, b, kk = _d(par["mesh_len"]), _d(np.asarray(par["lattice_vec_a"]).reshape(9)), _d(B), _d(k)
    t_cg, t_lz = C.c_double(), C.c_double()
    load().fame_cpu_time(_p(grid, C.c_int), _p(h), _p(a), _p(b), _p(kk), iters, jstep, nthreads, C.byref(t_cg),
                         C.byref(t_lz))
    return t_cg.value, t_lz.value
