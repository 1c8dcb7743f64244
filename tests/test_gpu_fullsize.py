"""Full-size configurations on the GPU against the reference's FP64 CUDA build run
on a B200 (tests/golden/*_ref.json made by make_golden.py ref-big):

  * the 96^3 simple-cubic band path (20 k-points, 10 bands) at the reference's
    default tolerances 1e-12: mixed precision within 1e-6 of the reference's
    frequencies and every band's relative residual <= 1e-6; FP64 within 1e-8 on
    four k-points;
  * FCC 64x55x52 (3 k-points, 10 bands), BCC 48x45x39 (3 k-points, 12 bands) and
    hexagonal 128x107x92 (2 k-points, 16 bands) at 1e-10: FP64 within 1e-8 and
    mixed within 1e-6 of the reference.
"""
import numpy as np
import pytest

import fame_b200 as fb
from fixtures import load_pre, load_ref

pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _ctx(par):
    ctx = fb.Context.from_par(par)
    ctx.set_material(par["binout"], par["material_num"], par["eps_in"], par["eps_out"])
    return ctx


def _ref(fix):
    ref = load_ref(fix)
    k = np.array([r["wave_vec"] for r in ref["kpoints"]])
    f = np.array([r["freq"] for r in ref["kpoints"]])
    es = np.array([r["es_iter"] for r in ref["kpoints"]])
    return k, f, es, ref["tol"]


def _relerr(f, fr):
    nz = fr > 0
    assert np.all(f[~nz] == 0)
    return np.max(np.abs(f[nz] - fr[nz]) / fr[nz])


def _tols(tol):
    return dict(es_tol=tol, ls_tol=tol, es_maxit=100, ls_maxit=1000, nstep=40)


def test_metric_band_path_mixed_at_reference_default_tolerance():
    par = load_pre("sc96")
    k, fr, _, tol = _ref("sc96_t12")
    ctx = _ctx(par)
    out = ctx.solve(k, nwant=fr.shape[1], precision=fb.MIXED, **_tols(tol))
    assert out["rc"] == fb.OK
    assert _relerr(out["freq"], fr) < 1e-6
    assert np.all(out["relres"] < 1e-6)
    assert np.all(out["relerr"] < 1e-6)
    sub = [1, 3, 6, 18]
    o64 = ctx.solve(k[sub], nwant=fr.shape[1], precision=fb.FP64, **_tols(tol))
    assert _relerr(o64["freq"], fr[sub]) < 1e-8
    assert np.all(o64["relres"] < 1e-6)


@pytest.mark.parametrize("name", ["fcc64", "bcc48", "hex128"])
def test_general_lattices_full_size(name):
    par = load_pre(name)
    k, fr, es, tol = _ref(name)
    ctx = _ctx(par)
    out = ctx.solve(k, nwant=fr.shape[1], precision=fb.FP64, **_tols(tol))
    assert out["rc"] == fb.OK
    assert _relerr(out["freq"], fr) < 1e-8
    got_es = np.array([c["es_iter"] for c in out["counters"]])
    assert np.mean(got_es == es) >= 0.5, (got_es, es)
    mx = ctx.solve(k, nwant=fr.shape[1], precision=fb.MIXED, **_tols(tol))
    assert mx["rc"] == fb.OK
    assert _relerr(mx["freq"], fr) < 1e-6
    assert np.all(mx["relerr"] < 1e-6)


def test_batched_band_path_in_one_graph():
    """BCC 48x45x39: 60 k-points along Gamma-H-N-Gamma-P (15 per segment, segment
    end excluded, built from the reference's vertex list), 12 bands, mixed precision,
    all 60 k-points as one batch in one CUDA graph.  The Gamma, H and N points match
    the reference's frequencies; three interior k-points solved one at a time match
    the batched result (the slots of a batch do not interact)."""
    par = load_pre("bcc48")
    v = par["kpoints"]  # Gamma, H, N, Gamma, P, ... (the reference's path GHNGPH|PN)
    seg = [(v[0], v[1]), (v[1], v[2]), (v[2], v[3]), (v[3], v[4])]
    k = np.array([a + (b - a) * (i / 15.0) for a, b in seg for i in range(15)])
    _, fr, _, tol = _ref("bcc48")
    ctx = _ctx(par)
    out = ctx.solve(k, nwant=12, precision=fb.MIXED, batch=60, use_graph=1, **_tols(tol))
    assert out["rc"] == fb.OK
    assert np.all(out["relerr"] < 1e-6)
    # Gamma (0 and 45), H (15), N (30) against the reference's k 0, 1, 2
    for i, r in ((0, 0), (15, 1), (30, 2), (45, 0)):
        assert _relerr(out["freq"][i:i + 1], fr[r:r + 1]) < 1e-6, i
    sub = [7, 22, 52]
    one = ctx.solve(k[sub], nwant=12, precision=fb.MIXED, batch=1, use_graph=1, **_tols(tol))
    assert np.max(np.abs(one["freq"] - out["freq"][sub]) / out["freq"][sub]) < 1e-10
