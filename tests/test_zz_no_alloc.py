"""fame_qbq_static (FP64 Q_r^* B^-1 Q_r with its scratch in a static device array,
no allocation, no context) against fame_apply(FAME_OP_QBQ, FAME_FP64) through the
C ABI, on two calls in a row (the second reuses the scratch the first left behind).

Tolerance: 1e-12 relative (norm-wise), the FP64 operator bar; the two paths differ
only in where the scratch lives and in the rounding of the twiddle tables.
Collected last so that it also runs after every other test in one process.
"""
import ctypes as C

import numpy as np
import pytest

import fame_b200 as fb
from fixtures import edge_eps, load_apply, load_pre


def _lattice(par):
    return fb.make_lattice(par["grid"], par["mesh_len"], par["lattice_vec_a"], par["simple"], par["m"], par["t1"])


def test_oversized_grid_is_rejected_before_any_device_call():
    lib = fb.load()
    lat = fb.make_lattice((64, 64, 64), [1 / 64] * 3, [1, 0, 0, 0, 1, 0, 0, 0, 1], True)
    k = np.zeros(3)
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.fame_qbq_static(C.byref(lat), k.ctypes.data_as(C.POINTER(C.c_double)), dummy, dummy, dummy, None)
    assert rc == fb.ERR_UNSUPPORTED
    msg = lib.fame_last_error().decode()
    assert "262144 points" in msg and str(fb.QBQ_STATIC_SCRATCH_BYTES) in msg


def test_null_arguments_are_rejected():
    lib = fb.load()
    assert lib.fame_qbq_static(None, None, None, None, None, None) == fb.ERR_BAD_INPUT


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sc16", "fcc16", "bcc12", "hex12"])
def test_static_scratch_qbq_matches_context_qbq(name):
    torch = pytest.importorskip("torch")
    par = load_pre(name)
    N = par["N"]
    ctx = fb.Context.from_par(par)
    ctx.set_material(par["binout"], par["material_num"], par["eps_in"], par["eps_out"])
    inv_b = torch.from_numpy(1.0 / edge_eps(par)).to("cuda", torch.float64)
    lat = _lattice(par)
    rng = np.random.default_rng(5)
    # two calls in a row: a general k-point (Nd = N), then the Gamma point (Nd = N - 1)
    for k in (par["kpoints"][1], np.zeros(3)):
        nd = N - 1 if np.linalg.norm(k) == 0 else N
        x = rng.standard_normal(2 * nd) + 1j * rng.standard_normal(2 * nd)
        xd = torch.from_numpy(x).to("cuda")
        y_static = torch.full((2 * nd,), np.nan, dtype=torch.complex128, device="cuda")
        y_ctx = torch.zeros(2 * nd, dtype=torch.complex128, device="cuda")
        fb.qbq_static(lat, k, inv_b, xd, y_static)
        torch.cuda.synchronize()
        assert ctx.apply(fb.OP_QBQ, k, xd, y_ctx, fb.FP64) == nd
        a, b = y_static.cpu().numpy(), y_ctx.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12


@pytest.mark.gpu
def test_static_scratch_qbq_prime_axis_lengths():
    """A 23 x 19 x 34 simple-cubic grid (prime factors 23, 19, 17: the prime-pass
    kernels) with a random 1/eps, against the context's FP64 QBQ."""
    torch = pytest.importorskip("torch")
    grid = (23, 19, 34)
    N = int(np.prod(grid))
    par = dict(grid=grid, mesh_len=[1.0 / g for g in grid], lattice_vec_a=[1, 0, 0, 0, 1, 0, 0, 0, 1],
               simple=True, m=(0, 0, 0, 0), t1=np.zeros(3))
    ctx = fb.Context.from_par(par)
    rng = np.random.default_rng(17)
    B = rng.uniform(1.0, 13.0, 3 * N)
    ctx.set_eps(B)
    inv_b = torch.from_numpy(1.0 / B).to("cuda", torch.float64)
    lat = _lattice(par)
    k = np.array([0.3, -0.2, 0.45])
    x = rng.standard_normal(2 * N) + 1j * rng.standard_normal(2 * N)
    xd = torch.from_numpy(x).to("cuda")
    y_static = torch.full((2 * N,), np.nan, dtype=torch.complex128, device="cuda")
    y_ctx = torch.zeros(2 * N, dtype=torch.complex128, device="cuda")
    fb.qbq_static(lat, k, inv_b, xd, y_static)
    torch.cuda.synchronize()
    assert ctx.apply(fb.OP_QBQ, k, xd, y_ctx, fb.FP64) == N
    a, b = y_static.cpu().numpy(), y_ctx.cpu().numpy()
    assert np.all(np.isfinite(a))
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12


@pytest.mark.gpu
def test_static_scratch_qbq_matches_reference_fixture():
    torch = pytest.importorskip("torch")
    par = load_pre("sc16")
    ap = load_apply("sc16")
    inv_b = torch.from_numpy(1.0 / edge_eps(par)).to("cuda", torch.float64)
    lat = _lattice(par)
    for kidx in (0, 1):
        nd = int(ap[f"Nd_{kidx}"])
        x = torch.from_numpy(np.ascontiguousarray(ap["x"][: 2 * nd])).to("cuda")
        y = torch.zeros(2 * nd, dtype=torch.complex128, device="cuda")
        fb.qbq_static(lat, par["kpoints"][kidx], inv_b, x, y)
        torch.cuda.synchronize()
        ref = ap[f"QBQ_{kidx}"]
        assert np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-12
