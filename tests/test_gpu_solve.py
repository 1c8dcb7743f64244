"""Full band-structure solves on the GPU against the reference's FP64 CUDA build.

Bars (eigenvalues within relative 1e-6 at residual 1e-6):
  * FP64 path: frequencies within 1e-8 relative of the reference, same number of
    A_r^-1 applications (same Lanczos path);
  * mixed path (FP32 operator/CG + FP64 refinement, FP64 Lanczos): within 1e-6;
  * relative residual ||C^H C E - w^2 B E|| / (w^2 ||B E||) <= 1e-6, checked with
    the oracle's independent sparse curl on the returned eigenvectors.
"""
import numpy as np
import pytest

import fame_b200 as fb
import fame_oracle as fo
from fixtures import edge_eps, load_pre, load_ref

pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = dict(es_tol=1e-10, ls_tol=1e-10, es_maxit=100, ls_maxit=1000, nstep=40)


def _ctx(par):
    ctx = fb.Context.from_par(par)
    ctx.set_material(par["binout"], par["material_num"], par["eps_in"], par["eps_out"])
    return ctx


def _ref(name):
    ref = load_ref(name)
    k = np.array([r["wave_vec"] for r in ref["kpoints"]])
    f = np.array([r["freq"] for r in ref["kpoints"]])
    es = np.array([r["es_iter"] for r in ref["kpoints"]])
    return k, f, es


def _relerr(f, fr):
    nz = fr > 0
    assert np.all(f[~nz] == 0)
    return np.max(np.abs(f[nz] - fr[nz]) / fr[nz])


@pytest.mark.parametrize("name", ["sc16", "fcc16", "bcc12", "hex12"])
def test_fp64_matches_reference(name):
    par = load_pre(name)
    k, fr, es = _ref(name)
    ctx = _ctx(par)
    out = ctx.solve(k, nwant=fr.shape[1], precision=fb.FP64, **TOL)
    assert out["rc"] == fb.OK
    assert _relerr(out["freq"], fr) < 1e-8
    assert np.all(out["relres"] < 1e-6)
    got_es = np.array([c["es_iter"] for c in out["counters"]])
    assert np.mean(got_es == es) >= 0.8, (got_es, es)


@pytest.mark.parametrize("name", ["sc16", "fcc16", "bcc12", "hex12"])
def test_mixed_matches_reference(name):
    par = load_pre(name)
    k, fr, _ = _ref(name)
    ctx = _ctx(par)
    out = ctx.solve(k, nwant=fr.shape[1], precision=fb.MIXED, **TOL)
    assert out["rc"] == fb.OK
    assert _relerr(out["freq"], fr) < 1e-6
    assert np.all(out["relres"] < 1e-6)
    assert np.all(out["relerr"] < 1e-6)


def test_graph_and_host_driven_agree_and_batches_are_independent():
    par = load_pre("sc16")
    k, fr, _ = _ref("sc16")
    ctx = _ctx(par)
    a = ctx.solve(k[:4], nwant=10, precision=fb.FP64, use_graph=1, batch=4, **TOL)
    b = ctx.solve(k[:4], nwant=10, precision=fb.FP64, use_graph=0, batch=4, **TOL)
    c = ctx.solve(k[:4], nwant=10, precision=fb.FP64, use_graph=1, batch=1, **TOL)
    assert np.array_equal(a["freq"], b["freq"])
    assert np.max(np.abs(a["freq"] - c["freq"])) < 1e-12


def test_concurrent_lanes_match_a_single_batch():
    """An automatic batch of 8 or more k-points runs as two concurrent lanes (contiguous
    blocks, one lane context each); the option lanes = 1 solves them as one batch.  Both
    give the reference's frequencies and agree to 1e-12; a permittivity change reaches
    the lane contexts."""
    par = load_pre("sc16")
    k, fr, _ = _ref("sc16")
    idx = np.arange(8) % len(k)
    ctx = _ctx(par)
    assert ctx.get_option("lanes") == 2
    two = ctx.solve(k[idx], nwant=10, precision=fb.MIXED, **TOL)
    ctx.set_option("lanes", 1)
    one = ctx.solve(k[idx], nwant=10, precision=fb.MIXED, **TOL)
    assert two["rc"] == fb.OK and one["rc"] == fb.OK
    assert _relerr(two["freq"], fr[idx]) < 1e-6
    assert np.max(np.abs(two["freq"] - one["freq"]) / np.maximum(one["freq"], 1e-300)) < 1e-12
    # a new permittivity (uniform 2) reaches every lane: all k-points see the same medium
    ctx.set_option("lanes", 2)
    ctx.set_eps(np.full(3 * par["N"], 2.0))
    u2 = ctx.solve(k[idx], nwant=10, precision=fb.MIXED, **TOL)
    ctx.set_option("lanes", 1)
    u1 = ctx.solve(k[idx], nwant=10, precision=fb.MIXED, **TOL)
    assert np.max(np.abs(u2["freq"] - u1["freq"]) / np.maximum(u1["freq"], 1e-300)) < 1e-12
    assert np.max(np.abs(u2["freq"] - two["freq"])) > 1e-3


def test_eigenvectors_satisfy_the_curl_equation():
    """Independent check: sparse curl (FAME_Matrix_Curl.cpp semantics) on E."""
    par = load_pre("sc16")
    k, fr, _ = _ref("sc16")
    ctx = _ctx(par)
    B = edge_eps(par)
    for prec in (fb.FP64, fb.MIXED):
        out = ctx.solve(k[1:3], nwant=10, precision=prec, want_vectors=1, **TOL)
        for q in range(2):
            for i in range(10):
                r = fo.relative_residual_simple(out["evec"][q, i], out["freq"][q, i], k[1 + q], par, B)
                assert r < 1e-6
                assert abs(r - out["relres"][q, i]) <= 0.05 * r + 1e-12


def test_gamma_point_patch():
    par = load_pre("sc16")
    k, fr, _ = _ref("sc16")
    ctx = _ctx(par)
    out = ctx.solve(k[:1], nwant=10, precision=fb.FP64, want_vectors=1, **TOL)
    assert out["counters"][0]["Nd"] == par["N"] - 1
    assert out["freq"][0, 0] == 0 and out["freq"][0, 1] == 0
    v = 1.0 / np.sqrt(3 * par["N"])
    assert np.allclose(out["evec"][0, 0], v) and np.allclose(out["evec"][0, 1], v)


@pytest.mark.parametrize("precision,tol", [(fb.FP64, 1e-8), (fb.MIXED, 1e-6)])
def test_hexagonal_gamma_matches_an_independent_eigensolver(precision, tol):
    """Hexagonal 36x30x26 (the hex 128 crystal on a grid an independent solver can
    handle), at the path's two Gamma points: the two zero bands, then every band up to
    the 14th of ARPACK's spectrum of A_r (tests/golden/hex36_gamma_oracle.json,
    seeded random start on the oracle's A_r^-1), degenerate pairs included."""
    import json
    import os
    par = load_pre("hex36")
    with open(os.path.join(os.path.dirname(__file__), "golden", "hex36_gamma_oracle.json")) as f:
        orc = json.load(f)
    ctx = _ctx(par)
    k = par["kpoints"][orc["gamma_kidx"]]
    out = ctx.solve(k, nwant=16, precision=precision, **TOL)
    assert out["rc"] == fb.OK
    ref = np.array(orc["freq"][:14])
    for row, c in zip(out["freq"], out["counters"]):
        assert c["Nd"] == par["N"] - 1
        assert row[0] == 0 and row[1] == 0
        assert np.max(np.abs(row[2:] - ref) / ref) < tol
    assert np.all(out["relres"][:, 2:] < 1e-6)
    ctx.close()


def test_hexagonal_vertices_match_the_oracle():
    """Hexagonal 36x30x26, the M, K and A vertices (tests/golden/hex36_oracle.json: the
    oracle's FP64 restatement of the reference's solver at 1e-10): FP64 within 1e-8 and
    mixed precision within 1e-6, with every band's relative residual below 1e-6.  The
    grid's axes (36 = 4 x 9, 30 = 2 x 3 x 5, 26 = 2 x 13) run the runtime-geometry plans."""
    import json
    import os
    par = load_pre("hex36")
    with open(os.path.join(os.path.dirname(__file__), "golden", "hex36_oracle.json")) as f:
        orc = json.load(f)
    k = np.array([r["wave_vec"] for r in orc["kpoints"]])
    fr = np.array([r["freq"] for r in orc["kpoints"]])
    ctx = _ctx(par)
    for precision, tol in ((fb.FP64, 1e-8), (fb.MIXED, 1e-6)):
        out = ctx.solve(k, nwant=orc["nwant"], precision=precision, **TOL)
        assert out["rc"] == fb.OK
        assert _relerr(out["freq"], fr) < tol, precision
        assert np.all(out["relres"] < 1e-6)
    ctx.close()


def test_precision_and_batch_changes_on_one_context():
    """One context grows its batch in mixed precision (1 then 3 k-points) and then
    solves the same 3 k-points in FP64: every workspace buffer follows the largest
    batch seen, whichever precision asked for it."""
    par = load_pre("sc16")
    k, fr, _ = _ref("sc16")
    ctx = _ctx(par)
    ctx.solve(k[:1], nwant=10, precision=fb.MIXED, **TOL)
    mx = ctx.solve(k[1:4], nwant=10, precision=fb.MIXED, **TOL)
    f64 = ctx.solve(k[1:4], nwant=10, precision=fb.FP64, **TOL)
    assert mx["rc"] == fb.OK and f64["rc"] == fb.OK
    assert _relerr(mx["freq"], fr[1:4]) < 1e-6
    assert _relerr(f64["freq"], fr[1:4]) < 1e-8
