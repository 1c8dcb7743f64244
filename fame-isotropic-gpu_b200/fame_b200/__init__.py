"""Python binding of the FAME B200 band-structure library (include/fame_b200.h).

The compute path is the CUDA library libfame_b200.so built in-tree
(fame-isotropic-gpu_b200/Makefile).  This module only marshals arguments through
ctypes; there is no Python or CPU fallback: if the library or a CUDA device is
missing, the calls raise.

Mirrors the reference's interface for the path (paths relative to its project root):
  - Context.solve      <- FAME_Fast_Algorithms_Driver over the k-loop of FAME_Main_Code
                          (FAME_Main/FAME_Main_Code.cu:79-171)
  - Context.apply      <- FAME_Matrix_Vector_Production_{Qr,Qrs,Pr,Prs,Isotropic_QBQ,
                          Isotropic_invAr}
  - Context.set_material <- FAME_Matrix_B_Isotropic (FAME_Main/FAME_Matrix_B_Isotropic.cu)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_HERE, "libfame_b200.so")

OK, ERR_BAD_INPUT, ERR_NO_CONVERGENCE, ERR_WATCHDOG, ERR_CUDA, ERR_NO_DEVICE, ERR_UNSUPPORTED, ERR_IO = range(8)
FP64, MIXED = 0, 1
OP_QR, OP_QRS, OP_QBQ, OP_PR, OP_PRS, OP_INVAR = range(6)

# every symbol declared in include/fame_b200.h
EXPORTS = ("fame_ctx_create", "fame_ctx_destroy", "fame_set_eps", "fame_set_material", "fame_solve_kpoints",
           "fame_apply", "fame_adjoint", "fame_ctx_sizes", "fame_last_error", "fame_version", "fame_ctx_stream",
           "fame_launch_count", "fame_bench_qbq", "fame_qbq_static", "fame_material_locate",
           "fame_write_eigenvectors", "fame_writer_start", "fame_writer_finish", "fame_set_loop_cap",
           "fame_bench_cg", "fame_set_eps_device", "fame_adjoint_vjp", "fame_set_option", "fame_get_option",
           "fame_tune")
# fame_kcounters.detail bits (FAME_KSTATUS_*)
KSTATUS_QL, KSTATUS_LANCZOS, KSTATUS_CG = 1, 2, 4
QBQ_STATIC_SCRATCH_BYTES = 4 << 20  # FAME_QBQ_STATIC_SCRATCH_BYTES


class FameError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fame error {code}: {msg}")
        self.code = code


class Lattice(C.Structure):
    _fields_ = [("grid", C.c_int * 3), ("mesh_len", C.c_double * 3), ("lattice_vec_a", C.c_double * 9),
                ("simple", C.c_int), ("m", C.c_int * 4), ("t1", C.c_double * 3)]


class SolverParams(C.Structure):
    _fields_ = [("nwant", C.c_int), ("nstep", C.c_int), ("es_maxit", C.c_int), ("es_tol", C.c_double),
                ("ls_maxit", C.c_int), ("ls_tol", C.c_double), ("precision", C.c_int), ("batch", C.c_int),
                ("use_graph", C.c_int), ("inner_tol", C.c_double), ("inner_maxit", C.c_int),
                ("want_vectors", C.c_int)]


class LocateGeometry(C.Structure):
    _fields_ = [("grid", C.c_int * 3), ("mesh_len", C.c_double * 3), ("lattice_vec_a", C.c_double * 9),
                ("Omega", C.c_double * 9), ("permutation", C.c_int * 3)]


class MaterialShapes(C.Structure):
    _fields_ = [("material_num", C.c_int), ("sphere_num", C.POINTER(C.c_int)),
                ("sphere_centers", C.POINTER(C.c_double)), ("sphere_radius", C.POINTER(C.c_double)),
                ("cylinder_num", C.POINTER(C.c_int)), ("cylinder_top_centers", C.POINTER(C.c_double)),
                ("cylinder_bot_centers", C.POINTER(C.c_double)), ("cylinder_radius", C.POINTER(C.c_double))]


class KCounters(C.Structure):
    _fields_ = [("ls_iter", C.c_int), ("es_iter", C.c_int), ("restarts", C.c_int), ("status", C.c_int),
                ("Nd", C.c_int), ("refine", C.c_int), ("detail", C.c_int)]


_lib = None


def load():
    """Loads libfame_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FameError(ERR_UNSUPPORTED, f"{LIB_PATH} not built (run __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.fame_ctx_create.argtypes = [C.c_int, C.POINTER(Lattice), C.POINTER(P)]
    lib.fame_ctx_destroy.argtypes = [P]
    lib.fame_ctx_destroy.restype = None
    lib.fame_set_eps.argtypes = [P, D]
    lib.fame_set_material.argtypes = [P, C.POINTER(C.c_int), C.c_int, D, C.c_double]
    lib.fame_solve_kpoints.argtypes = [P, D, C.c_int, C.POINTER(SolverParams), D, D, D, D, D, C.POINTER(KCounters)]
    lib.fame_apply.argtypes = [P, C.c_int, D, P, P, C.c_int, C.POINTER(SolverParams), C.POINTER(C.c_int)]
    lib.fame_adjoint.argtypes = [P, D, D, C.c_int, C.c_int, D]
    lib.fame_ctx_sizes.argtypes = [P, C.POINTER(C.c_longlong)]
    lib.fame_ctx_stream.argtypes = [P]
    lib.fame_ctx_stream.restype = C.c_void_p
    lib.fame_launch_count.argtypes = [P, C.POINTER(C.c_ulonglong)]
    lib.fame_bench_qbq.argtypes = [P, D, C.c_int, C.c_int, C.c_int, D, D]
    lib.fame_qbq_static.argtypes = [C.POINTER(Lattice), D, P, P, P, P]
    lib.fame_material_locate.argtypes = [C.c_int, C.POINTER(LocateGeometry), C.POINTER(MaterialShapes),
                                         C.POINTER(C.c_int)]
    lib.fame_write_eigenvectors.argtypes = [C.c_char_p, D, C.c_int, C.c_longlong, C.c_int, C.c_int]
    lib.fame_writer_start.argtypes = [C.c_char_p, D, C.c_int, C.c_longlong, C.c_int, C.c_int, C.POINTER(P)]
    lib.fame_writer_finish.argtypes = [P]
    lib.fame_set_loop_cap.argtypes = [P, C.c_int]
    lib.fame_bench_cg.argtypes = [P, D, C.c_int, C.c_int, D, D]
    lib.fame_set_eps_device.argtypes = [P, P]
    lib.fame_adjoint_vjp.argtypes = [P, C.c_int, D, D, C.c_int, C.c_double, P]
    lib.fame_set_option.argtypes = [P, C.c_char_p, C.c_int]
    lib.fame_get_option.argtypes = [P, C.c_char_p, C.POINTER(C.c_int)]
    lib.fame_tune.argtypes = [P, D, C.c_int, C.c_int, C.c_char_p, C.c_char_p, C.c_int]
    lib.fame_last_error.restype = C.c_char_p
    lib.fame_version.restype = C.c_char_p
    for fn in ("fame_ctx_create", "fame_set_eps", "fame_set_material", "fame_solve_kpoints", "fame_apply",
               "fame_adjoint", "fame_ctx_sizes", "fame_launch_count", "fame_bench_qbq", "fame_qbq_static",
               "fame_material_locate", "fame_write_eigenvectors", "fame_writer_start", "fame_writer_finish",
               "fame_set_loop_cap", "fame_bench_cg", "fame_set_eps_device", "fame_adjoint_vjp",
               "fame_set_option", "fame_get_option", "fame_tune"):
        getattr(lib, fn).restype = C.c_int
    _lib = lib
    return lib


def _check(rc):
    if rc != OK:
        raise FameError(rc, load().fame_last_error().decode())


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def reduced_size(lattice, k):
    """Nd of wave vector k on `lattice` (a Lattice): N - 1 at the Gamma point (|k| below
    1e-4 for Simple lattices, 1e-3 for General ones, FAME_Main/FAME_Matrix_Lambdas.cu:157
    and :406), else N.  The same rule as the library's."""
    N = int(lattice.grid[0]) * int(lattice.grid[1]) * int(lattice.grid[2])
    kk = np.asarray(k, dtype=np.float64).reshape(-1)
    if kk.size != 3:
        raise ValueError("k must have 3 components")
    return N - 1 if float(np.sqrt(np.sum(kk * kk))) < (1e-4 if lattice.simple else 1e-3) else N


def _check_device_tensor(t, name, dtype, numel, device):
    """Raises ValueError unless t is a contiguous CUDA tensor of `dtype` with exactly
    `numel` elements on CUDA device `device` (None: the current device): the library
    reads and writes exactly that many elements at t.data_ptr(), so anything else
    would run out of bounds."""
    import torch
    if not isinstance(t, torch.Tensor):
        raise ValueError(f"{name} must be a torch tensor")
    if t.device.type != "cuda":
        raise ValueError(f"{name} must be a CUDA tensor (got {t.device})")
    if device is None:
        device = torch.cuda.current_device()
    if t.device.index != device:
        raise ValueError(f"{name} must be on cuda:{device} (got {t.device})")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype} (got {t.dtype})")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.numel() != numel:
        raise ValueError(f"{name} must have {numel} elements (got {t.numel()})")


def make_lattice(grid, mesh_len, lattice_vec_a, simple, m=(0, 0, 0, 0), t1=(0.0, 0.0, 0.0)):
    L = Lattice()
    L.grid[:] = [int(v) for v in grid]
    L.mesh_len[:] = [float(v) for v in mesh_len]
    L.lattice_vec_a[:] = [float(v) for v in lattice_vec_a]
    L.simple = int(bool(simple))
    L.m[:] = [int(v) for v in m]
    L.t1[:] = [float(v) for v in t1]
    return L


def solver_params(nwant=10, nstep=40, es_maxit=100, es_tol=1e-10, ls_maxit=1000, ls_tol=1e-10,
                  precision=FP64, batch=0, use_graph=1, inner_tol=0.0, inner_maxit=0, want_vectors=0):
    p = SolverParams()
    p.nwant, p.nstep, p.es_maxit, p.es_tol = nwant, nstep, es_maxit, es_tol
    p.ls_maxit, p.ls_tol, p.precision, p.batch = ls_maxit, ls_tol, precision, batch
    p.use_graph, p.inner_tol, p.inner_maxit, p.want_vectors = use_graph, inner_tol, inner_maxit, want_vectors
    return p


class Context:
    """One device, one grid/lattice, one permittivity field."""

    def __init__(self, grid, mesh_len, lattice_vec_a, simple, m=(0, 0, 0, 0), t1=(0.0, 0.0, 0.0), device=0):
        lib = load()
        self._lat = make_lattice(grid, mesh_len, lattice_vec_a, simple, m, t1)
        self.N = int(np.prod(grid))
        self.device = int(device)
        h = C.c_void_p()
        _check(lib.fame_ctx_create(device, C.byref(self._lat), C.byref(h)))
        self._h = h

    @classmethod
    def from_par(cls, par, device=0):
        return cls(par["grid"], par["mesh_len"], par["lattice_vec_a"], par["simple"], par["m"], par["t1"], device)

    def close(self):
        if getattr(self, "_h", None):
            load().fame_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_eps(self, B):
        B = np.ascontiguousarray(B, dtype=np.float64)
        assert B.size == 3 * self.N
        _check(load().fame_set_eps(self._h, _dptr(B)))

    def set_eps_device(self, B):
        """Edge permittivities from a contiguous float64 CUDA tensor of 3N values on the
        context's device (stays on the GPU)."""
        import torch
        _check_device_tensor(B, "B", torch.float64, 3 * self.N, self.device)
        _check(load().fame_set_eps_device(self._h, C.c_void_p(B.data_ptr())))

    def set_material(self, binout, material_num, eps_in, eps_out):
        b = np.ascontiguousarray(binout, dtype=np.int32)
        e = np.ascontiguousarray(eps_in, dtype=np.float64)
        _check(load().fame_set_material(self._h, b.ctypes.data_as(C.POINTER(C.c_int)), int(material_num),
                                        _dptr(e), float(eps_out)))

    def solve(self, kpoints, params=None, resabs=False, vectors_on_device=False, **kw):
        """Returns dict(freq, relres, relerr, counters[, resabs][, evec]) for kpoints (nk, 3).
        resabs: also the residual norm of E scaled as the reference restores it.
        vectors_on_device: keep the eigenvectors on the GPU (for adjoint_vjp) instead of
        returning them; all k-points then run as one batch."""
        p = params or solver_params(**kw)
        if vectors_on_device:
            q = SolverParams()
            C.memmove(C.byref(q), C.byref(p), C.sizeof(SolverParams))
            q.want_vectors = 1
            p = q
        self.solves = getattr(self, "solves", 0) + 1
        k = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        nk = k.shape[0]
        freq = np.zeros((nk, p.nwant))
        rr = np.zeros((nk, p.nwant))
        re = np.zeros((nk, p.nwant))
        ev = np.zeros((nk, p.nwant, 3 * self.N), dtype=np.complex128) if p.want_vectors and not vectors_on_device \
            else None
        cnt = (KCounters * nk)()
        ra = np.zeros((nk, p.nwant)) if resabs else None
        rc = load().fame_solve_kpoints(self._h, _dptr(k), nk, C.byref(p), _dptr(freq), _dptr(rr), _dptr(re),
                                       _dptr(ra) if ra is not None else None,
                                       ev.ctypes.data_as(C.POINTER(C.c_double)) if ev is not None else None, cnt)
        out = dict(freq=freq, relres=rr, relerr=re, rc=rc,
                   counters=[dict(ls_iter=c.ls_iter, es_iter=c.es_iter, restarts=c.restarts, status=c.status,
                                  Nd=c.Nd, refine=c.refine, detail=c.detail) for c in cnt])
        if ev is not None:
            out["evec"] = ev
        if ra is not None:
            out["resabs"] = ra
        if rc not in (OK, ERR_NO_CONVERGENCE):
            _check(rc)
        return out

    def apply(self, op, k, x, y, precision=FP64, params=None):
        """Applies operator `op` at wave vector k to device buffers x -> y (contiguous
        torch CUDA tensors on the context's device, complex128 for FP64 / complex64 for
        MIXED; reduced vectors have 2*Nd elements, fields 3N).  Returns Nd.  Raises
        ValueError on a tensor of the wrong device, type, layout or size."""
        import torch
        kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
        Nd = reduced_size(self._lat, kk)
        dt = torch.complex128 if precision == FP64 else torch.complex64
        n_in = 3 * self.N if op in (OP_QRS, OP_PRS) else 2 * Nd
        n_out = 3 * self.N if op in (OP_QR, OP_PR) else 2 * Nd
        _check_device_tensor(x, "x", dt, n_in, self.device)
        _check_device_tensor(y, "y", dt, n_out, self.device)
        nd = C.c_int()
        p = params or solver_params()
        _check(load().fame_apply(self._h, int(op), _dptr(kk), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                 int(precision), C.byref(p), C.byref(nd)))
        return nd.value

    def set_loop_cap(self, max_trips):
        """Bounds every device loop of later solves to max_trips trips (0: defaults);
        a loop that reaches it ends the solve with ERR_WATCHDOG."""
        _check(load().fame_set_loop_cap(self._h, int(max_trips)))

    def set_option(self, name, value):
        """Execution option of the context (fame_set_option)."""
        _check(load().fame_set_option(self._h, name.encode(), int(value)))

    def get_option(self, name):
        v = C.c_int()
        _check(load().fame_get_option(self._h, name.encode(), C.byref(v)))
        return v.value

    def tune(self, k, precision=MIXED, batch=1, cache_file=None):
        """FFT plan autotuner (fame_tune): times candidate plans, applies the fastest
        and returns it as text; cache_file keeps winners across runs."""
        kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
        buf = C.create_string_buffer(256)
        cf = None if cache_file is None else os.fsencode(cache_file)
        _check(load().fame_tune(self._h, _dptr(kk), int(precision), int(batch), cf, buf, 256))
        return buf.value.decode()

    def stream(self):
        """The context's cudaStream_t as an int (for torch.cuda.ExternalStream)."""
        return load().fame_ctx_stream(self._h)

    def launch_count(self):
        n = C.c_ulonglong()
        _check(load().fame_launch_count(self._h, C.byref(n)))
        return n.value

    def bench_qbq(self, k, precision=MIXED, reps=20, nbatch=1):
        """Mean device ms of one L2-cold Q_r^* B^-1 Q_r apply to a batch of nbatch
        vectors, and of its 3 stages."""
        kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
        ms = C.c_double()
        st = np.zeros(3)
        _check(load().fame_bench_qbq(self._h, _dptr(kk), int(precision), int(reps), int(nbatch), C.byref(ms),
                                     _dptr(st)))
        return ms.value, st

    def bench_cg(self, k, reps=20, nbatch=1):
        """Mean device ms of one FP32 CG iteration (its three kernels, L2 flushed
        before each) on a batch of nbatch k-points, and of each kernel."""
        kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
        ms = C.c_double()
        st = np.zeros(3)
        _check(load().fame_bench_cg(self._h, _dptr(kk), int(reps), int(nbatch), C.byref(ms), _dptr(st)))
        return ms.value, st

    def adjoint_vjp(self, kidx, freq, grad_w, rel_gap=1e-6, out=None):
        """sum_i grad_w[i] d(omega_i)/d(eps_voxel) as a float64 CUDA tensor (N,) on the
        context's device, for k-point kidx of the last solve(vectors_on_device=True).
        Degenerate groups (relative gap <= rel_gap) must carry equal weights."""
        import torch
        f = np.ascontiguousarray(freq, dtype=np.float64).reshape(-1)
        g = np.ascontiguousarray(grad_w, dtype=np.float64).reshape(-1)
        if f.size != g.size:
            raise ValueError("freq and grad_w differ in length")
        if out is None:
            out = torch.empty(self.N, dtype=torch.float64, device=f"cuda:{self.device}")
        _check_device_tensor(out, "out", torch.float64, self.N, self.device)
        _check(load().fame_adjoint_vjp(self._h, int(kidx), _dptr(f), _dptr(g), f.size, float(rel_gap),
                                       C.c_void_p(out.data_ptr())))
        return out

    def adjoint(self, freq, evec):
        """d(omega_i)/d(eps_voxel) for one k: freq (nwant,), evec (nwant, 3N) complex128 host."""
        f = np.ascontiguousarray(freq, dtype=np.float64)
        e = np.ascontiguousarray(evec, dtype=np.complex128)
        nw = f.size
        g = np.zeros((nw, self.N))
        _check(load().fame_adjoint(self._h, _dptr(f), e.ctypes.data_as(C.POINTER(C.c_double)), nw, 1, _dptr(g)))
        return g


def material_locate(grid, mesh_len, lattice_vec_a, Omega, permutation, material, device=0):
    """Binout (int32, 3 * material_num * N) on the GPU through fame_material_locate.
    material: dict with material_num, sphere_num, sphere_centers, sphere_radius,
    cylinder_num, cylinder_top_centers, cylinder_bot_centers, cylinder_radius."""
    g = LocateGeometry()
    g.grid[:] = [int(v) for v in grid]
    g.mesh_len[:] = [float(v) for v in mesh_len]
    g.lattice_vec_a[:] = [float(v) for v in lattice_vec_a]
    g.Omega[:] = [float(v) for v in Omega]
    g.permutation[:] = [int(v) for v in permutation]
    keep = []

    def arr(v, t):
        a = np.ascontiguousarray(np.asarray(v, dtype=t).reshape(-1))
        keep.append(a)
        ct = C.c_int if t == np.int32 else C.c_double
        return a.ctypes.data_as(C.POINTER(ct)) if a.size else None

    m = MaterialShapes()
    m.material_num = int(material["material_num"])
    m.sphere_num = arr(material["sphere_num"], np.int32)
    m.sphere_centers = arr(material["sphere_centers"], np.float64)
    m.sphere_radius = arr(material["sphere_radius"], np.float64)
    m.cylinder_num = arr(material["cylinder_num"], np.int32)
    m.cylinder_top_centers = arr(material["cylinder_top_centers"], np.float64)
    m.cylinder_bot_centers = arr(material["cylinder_bot_centers"], np.float64)
    m.cylinder_radius = arr(material["cylinder_radius"], np.float64)
    out = np.zeros(3 * m.material_num * int(np.prod(grid)), dtype=np.int32)
    _check(load().fame_material_locate(int(device), C.byref(g), C.byref(m), out.ctypes.data_as(C.POINTER(C.c_int))))
    return out


def qbq_static(lattice, k, inv_b, x, y, stream=0):
    """Q_r^* B^-1 Q_r in FP64 through fame_qbq_static (no device allocation, no
    context): lattice from make_lattice, inv_b (3N float64), x and y (2*Nd
    complex128) contiguous torch CUDA tensors on the current device; enqueued on
    `stream` (a cudaStream_t as int, 0 = legacy default stream), not synchronised.
    Raises ValueError on a tensor of the wrong device, type, layout or size."""
    import torch
    kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
    N = int(lattice.grid[0]) * int(lattice.grid[1]) * int(lattice.grid[2])
    Nd = reduced_size(lattice, kk)
    # the call runs on the current device (whose scratch array it uses)
    _check_device_tensor(inv_b, "inv_b", torch.float64, 3 * N, None)
    _check_device_tensor(x, "x", torch.complex128, 2 * Nd, None)
    _check_device_tensor(y, "y", torch.complex128, 2 * Nd, None)
    _check(load().fame_qbq_static(C.byref(lattice), _dptr(kk), C.c_void_p(inv_b.data_ptr()),
                                  C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(stream)))


def write_eigenvectors(evec, kidx, directory=None, nthreads=0):
    """Data_EV_<kk>_<bb>.txt files of one wave vector in the reference's format
    (FAME_Save_Eigenvector) through fame_write_eigenvectors: evec is (nwant, 3N)
    complex128 on the host, kidx the 0-based wave-vector index."""
    ev = np.ascontiguousarray(np.asarray(evec, dtype=np.complex128))
    if ev.ndim != 2:
        raise ValueError("evec must be (nwant, 3N)")
    d = None if directory is None else os.fsencode(directory)
    _check(load().fame_write_eigenvectors(d, ev.ctypes.data_as(C.POINTER(C.c_double)), ev.shape[0], ev.shape[1],
                                          int(kidx), int(nthreads)))


def version():
    return load().fame_version().decode()
