"""Failure paths of the C ABI on the GPU: every case returns a status and none spins.

The reference only prints when a linear solve or Lanczos stops unconverged
(FAME_Main/CG.cu:81-84, FAME_Main/Lanczos_Isotropic.cu:84-85) and never checks the
permittivities it divides by (FAME_Main/FAME_Matrix_B_Isotropic.cu:62-66).  Here:
  - a NaN, zero or negative permittivity is FAME_ERR_BAD_INPUT;
  - an A_r^-1 solve that stops above ls_tol sets FAME_KSTATUS_CG on its k-point and
    the call returns FAME_ERR_NO_CONVERGENCE (FP64: ls_maxit = 1; mixed: one FP32
    product per inner solve, so the refinement cap is reached);
  - Lanczos without restarts (es_maxit = 0) at a tight tolerance sets
    FAME_KSTATUS_LANCZOS;
  - a loop bound set with fame_set_loop_cap that the CG loop reaches ends the solve
    with FAME_ERR_WATCHDOG, and the context stays usable afterwards;
  - solve arguments out of range (no k-points, a non-finite wave vector, band and
    step counts, tolerances, precision, no permittivity yet) are FAME_ERR_BAD_INPUT.
All inputs are host-side; no kernel is made to fault or hang."""
import numpy as np
import pytest

import fame_b200 as fb
from fixtures import edge_eps, load_pre, load_ref

pytestmark = pytest.mark.gpu


def _ctx(name="sc16"):
    par = load_pre(name)
    ctx = fb.Context.from_par(par)
    ctx.set_material(par["binout"], par["material_num"], par["eps_in"], par["eps_out"])
    return par, ctx


@pytest.mark.parametrize("bad", [np.nan, 0.0, -2.0, np.inf])
def test_bad_permittivity_is_rejected(bad):
    par, ctx = _ctx()
    B = edge_eps(par)
    B[123] = bad
    with pytest.raises(fb.FameError) as e:
        ctx.set_eps(B)
    assert e.value.code == fb.ERR_BAD_INPUT
    assert "permittivity" in str(e.value)
    # the context keeps its previous permittivity and still solves
    k = par["kpoints"][1:2]
    out = ctx.solve(k, nwant=4, nstep=20, es_tol=1e-8, ls_tol=1e-8)
    assert out["rc"] == fb.OK
    ctx.close()


BAD_SOLVES = [
    ("no k-points", dict(k=np.zeros((0, 3)))),
    ("NaN wave vector", dict(k=np.array([[0.1, np.nan, 0.2]]))),
    ("infinite wave vector", dict(k=np.array([[np.inf, 0.0, 0.0]]))),
    ("nwant = nstep", dict(nwant=20, nstep=20)),
    ("nwant < 1", dict(nwant=0)),
    ("nstep above 64", dict(nstep=65)),
    ("zero Lanczos tolerance", dict(es_tol=0.0)),
    ("NaN CG tolerance", dict(ls_tol=np.nan)),
    ("ls_maxit < 1", dict(ls_maxit=0)),
    ("negative es_maxit", dict(es_maxit=-1)),
    ("unknown precision", dict(precision=7)),
]


@pytest.mark.parametrize("what,bad", BAD_SOLVES, ids=[b[0] for b in BAD_SOLVES])
def test_invalid_solve_arguments_are_rejected(what, bad):
    """Every argument fame_solve_kpoints rejects returns FAME_ERR_BAD_INPUT with a
    message, and the context then solves normally.  The reference has no such checks:
    its k-loop takes the Popt.txt values as they are (FAME_Main/FAME_Main_Code.cu:79-133)."""
    par, ctx = _ctx()
    bad = dict(bad)
    k = bad.pop("k", par["kpoints"][1:2])
    kw = dict(nwant=4, nstep=20, es_tol=1e-8, ls_tol=1e-8)
    kw.update(bad)
    with pytest.raises(fb.FameError) as e:
        ctx.solve(k, **kw)
    assert e.value.code == fb.ERR_BAD_INPUT, what
    assert str(e.value).split(": ", 1)[1]  # the library's message
    out = ctx.solve(par["kpoints"][1:2], nwant=4, nstep=20, es_tol=1e-8, ls_tol=1e-8)
    assert out["rc"] == fb.OK
    ctx.close()


BAD_LATTICES = [
    ("zero mesh length", dict(mesh_len=(0.0, 1 / 16, 1 / 16)), fb.ERR_BAD_INPUT),
    ("NaN mesh length", dict(mesh_len=(1 / 16, np.nan, 1 / 16)), fb.ERR_BAD_INPUT),
    ("infinite lattice vector", dict(lattice_vec_a=[np.inf] + [0.0] * 8), fb.ERR_BAD_INPUT),
    ("grid below 2", dict(grid=(16, 1, 16)), fb.ERR_BAD_INPUT),
    ("FP64 plane beyond one CTA", dict(grid=(200, 200, 4)), fb.ERR_UNSUPPORTED),
]


@pytest.mark.parametrize("what,bad,code", BAD_LATTICES, ids=[b[0] for b in BAD_LATTICES])
def test_invalid_lattice_is_rejected(what, bad, code):
    """fame_ctx_create checks the lattice before it allocates anything: grid dimensions
    of at least 2, finite positive mesh lengths, finite lattice vectors, and a plane
    that fits one CTA's shared memory."""
    par = load_pre("sc16")
    kw = dict(grid=par["grid"], mesh_len=par["mesh_len"], lattice_vec_a=par["lattice_vec_a"],
              simple=par["simple"], m=par["m"], t1=par["t1"])
    kw.update(bad)
    with pytest.raises(fb.FameError) as e:
        fb.Context(**kw)
    assert e.value.code == code, what


def test_solve_before_permittivity_is_rejected():
    par = load_pre("sc16")
    ctx = fb.Context.from_par(par)
    with pytest.raises(fb.FameError) as e:
        ctx.solve(par["kpoints"][1:2], nwant=4, nstep=20)
    assert e.value.code == fb.ERR_BAD_INPUT
    assert "permittivity" in str(e.value)
    ctx.close()


@pytest.mark.parametrize("precision", [fb.FP64, fb.MIXED])
def test_linear_solve_cap_reports_no_convergence(precision):
    par, ctx = _ctx()
    k = par["kpoints"][1:3]
    kw = dict(nwant=4, nstep=20, es_tol=1e-10, es_maxit=1, ls_tol=1e-12, precision=precision)
    if precision == fb.FP64:
        kw["ls_maxit"] = 1
    else:
        kw["inner_maxit"] = 1
    out = ctx.solve(k, **kw)
    assert out["rc"] == fb.ERR_NO_CONVERGENCE
    for c in out["counters"]:
        assert c["status"] == fb.ERR_NO_CONVERGENCE
        assert c["detail"] & fb.KSTATUS_CG
    assert "ls_tol" in fb.load().fame_last_error().decode()
    ctx.close()


def test_lanczos_without_restarts_reports_no_convergence():
    par, ctx = _ctx()
    ref = load_ref("sc16")
    # the reference restarts at least once on these k-points at 1e-10
    idx = [i for i, r in enumerate(ref["kpoints"]) if r["es_iter"] > 40][:2]
    assert idx
    k = par["kpoints"][idx]
    out = ctx.solve(k, nwant=10, nstep=40, es_tol=1e-12, es_maxit=0, ls_tol=1e-12)
    assert out["rc"] == fb.ERR_NO_CONVERGENCE
    for c in out["counters"]:
        assert c["detail"] & fb.KSTATUS_LANCZOS
        assert c["restarts"] == 0
    ctx.close()


@pytest.mark.parametrize("precision", [fb.FP64, fb.MIXED])
def test_loop_cap_ends_the_solve_with_watchdog(precision):
    par, ctx = _ctx()
    k = par["kpoints"][1:2]
    kw = dict(nwant=4, nstep=20, es_tol=1e-10, ls_tol=1e-10, precision=precision)
    ctx.set_loop_cap(3)  # the CG needs about 30 products per A_r^-1 at this tolerance
    with pytest.raises(fb.FameError) as e:
        ctx.solve(k, **kw)
    assert e.value.code == fb.ERR_WATCHDOG
    ctx.set_loop_cap(0)
    out = ctx.solve(k, **kw)
    assert out["rc"] == fb.OK
    assert out["relres"].max() < 1e-6
    with pytest.raises(fb.FameError):
        ctx.set_loop_cap(-1)
    ctx.close()


def test_a_failing_lane_ends_the_call_with_its_status():
    """Eight k-points run as two concurrent lanes; a loop cap that runs out in both lanes
    (lane contexts take the context's cap) ends the call with FAME_ERR_WATCHDOG and the
    lane's message, and the context and its lanes solve normally once the cap is lifted."""
    par, ctx = _ctx()
    idx = np.arange(8) % len(par["kpoints"])
    k = par["kpoints"][idx]
    kw = dict(nwant=4, nstep=20, es_tol=1e-10, ls_tol=1e-10, precision=fb.MIXED)
    assert ctx.get_option("lanes") == 2
    ctx.set_loop_cap(3)
    with pytest.raises(fb.FameError) as e:
        ctx.solve(k, **kw)
    assert e.value.code == fb.ERR_WATCHDOG
    assert "trip cap" in str(e.value)
    ctx.set_loop_cap(0)
    out = ctx.solve(k, **kw)
    assert out["rc"] == fb.OK
    assert out["relres"].max() < 1e-6
    ctx.close()
