"""Drop-in check of FAME_Main_Code: the reference's own Main.cpp, preprocessing and
output writers linked against libfame_b200.so through shim/FAME_Main_Code_b200.cpp
(fame-isotropic-gpu_b200/shim/_build/fame_b200_main), against the reference's
unmodified program (oracle/_ref/fame_ref_main) on the same Popt.txt and material
description.  Bars: |frequencies| in Data_Omega_array.txt within 1e-8
(FAME_B200_PRECISION=fp64) and 1e-6 (default mixed precision) of the reference's;
the sign marks of Check_Residual (a frequency is stored negated when its residual
exceeds 1e-10; each program tests its own residual, so a band at the threshold may
differ) agree for at least 90% of the FP64 entries, and the residuals both programs
print per band (the reference's CPU sparse product, this library's FP64 band
statistics) agree within a factor of 2 for at least 95% of the FP64 bands (within a
degenerate band group the Ritz vectors are any basis of the same subspace, so their
individual residuals differ; elsewhere they agree to about 1%); the Lanczos counts
of the FP64 run in Data_Profile.txt match the reference's for at least 80% of the
k-points.
Both programs are built from the reference sources in this container
(oracle/build_ref.sh, fame-isotropic-gpu_b200/shim/build_main.sh); the tests skip
where they are absent."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import ref_inputs as ri

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "fame-isotropic-gpu_b200", "shim", "_build", "fame_b200_main")
REFMAIN = os.path.join(ROOT, "oracle", "_ref", "fame_ref_main")


def _read_omega(path):
    cols, cur = [], None
    for line in open(path):
        if re.match(r"Freq_array\(:, \d+\) = \[", line):
            cur = []
        elif line.startswith("];") and cur is not None:
            cols.append(cur)
            cur = None
        elif cur is not None and line.strip():
            cur.append(float(line))
    return np.array(cols)


def _read_es_iter(path):
    rows = [l.split(",") for l in open(path) if re.match(r"\s*\d+,", l)]
    return np.array([int(r[3]) for r in rows])


def _read_residuals(stdout):
    pat = re.compile(r"Freq\(\s*\d+\) = +[-\d.]+, residual = ([-\d.]+e[-+]\d+)")
    return np.array([float(m.group(1)) for m in map(pat.search, stdout.splitlines()) if m])


def _run(prog, workdir, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([prog], cwd=workdir, env=e, capture_output=True, text=True, timeout=600)


def test_dropin_without_device_fails_loudly(tmp_path):
    if not os.path.exists(DROPIN):
        pytest.skip("fame_b200_main not built (needs the reference sources)")
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    d = ri.make_workdir("sc16", str(tmp_path / "w"))
    r = _run(DROPIN, d)
    assert "no CUDA device" in r.stderr
    assert not os.path.exists(os.path.join(d, "Data_Omega_array.txt"))


def test_dropin_too_few_permittivities_is_a_status_not_a_prompt(tmp_path):
    """Four materials and one inner permittivity in Popt.txt: the reference asks for the
    missing values on stdin (FAME_Main/FAME_Matrix_B_Isotropic.cu:13-24); the drop-in
    reports the error and returns before any device call, reading nothing from stdin
    (values offered there are ignored) and writing no frequencies."""
    if not os.path.exists(DROPIN):
        pytest.skip("fame_b200_main not built (needs the reference sources)")
    d = str(tmp_path / "w")
    build, nx, pn, _, eps_out, nw, ns = ri.WORKLOADS["bcc12"]
    ri.write_workdir(d, "Syn_bcc12", build(), nx, pn, [10.0], eps_out, nw, ns, 1e-10, 100, 1e-10, 1000)
    r = subprocess.run([DROPIN], cwd=d, input="9.0\n9.0\n9.0\n9.0\n", capture_output=True, text=True,
                       timeout=300)
    assert "1 inner permittivities given for 4 materials" in r.stderr
    assert "Please input" not in r.stdout
    assert not os.path.exists(os.path.join(d, "Data_Omega_array.txt"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sc16", "fcc16"])
def test_dropin_matches_reference_main(tmp_path, name):
    if not (os.path.exists(DROPIN) and os.path.exists(REFMAIN)):
        pytest.skip("fame_b200_main / fame_ref_main not built")
    base = ri.make_workdir(name, str(tmp_path / "base"))
    runs = {}
    for tag, prog, env in (("ref", REFMAIN, None), ("fp64", DROPIN, {"FAME_B200_PRECISION": "fp64"}),
                           ("mixed", DROPIN, None)):
        d = str(tmp_path / tag)
        shutil.copytree(base, d)
        r = _run(prog, d, env)
        assert r.returncode == 0, r.stderr[-2000:]
        runs[tag] = (_read_omega(os.path.join(d, "Data_Omega_array.txt")),
                     _read_es_iter(os.path.join(d, "Data_Profile.txt")), _read_residuals(r.stdout))
    ref, es_ref, res_ref = runs["ref"]
    assert ref.shape[0] >= 2
    a = np.abs(ref)
    nz = a > 0
    for tag, tol in (("fp64", 1e-8), ("mixed", 1e-6)):
        w = runs[tag][0]
        assert w.shape == ref.shape
        assert np.all(w[~nz] == 0)
        assert np.max(np.abs(np.abs(w[nz]) - a[nz]) / a[nz]) < tol, tag
    assert np.mean(np.sign(runs["fp64"][0][nz]) == np.sign(ref[nz])) >= 0.9
    assert np.mean(runs["fp64"][1] == es_ref) >= 0.8
    res = runs["fp64"][2]
    assert res.shape == res_ref.shape
    pos = res_ref > 0
    assert np.mean(np.abs(np.log(res[pos] / res_ref[pos])) < np.log(2.0)) >= 0.95


def _read_ev(path):
    pat = re.compile(r"\(\s*([-+\d.e]+)\) \+ \(\s*([-+\d.e]+) \* 1i\)")
    v = [complex(float(m.group(1)), float(m.group(2))) for m in map(pat.match, open(path)) if m]
    return np.array(v)


@pytest.mark.gpu
def test_dropin_saves_eigenvectors_in_batches(tmp_path):
    """"Save Eigen Vector" set: the drop-in solves the wave vectors in batches (two host
    buffers, one batch's Data_EV files written while the next batch solves) and, with
    FAME_B200_SAVE_BATCH=1, one wave vector per solve.  Both runs write one file per wave
    vector and band, with the same frequencies (to 1e-10) and the same fields: each
    batched field lies in the span of the one-at-a-time run's fields of its degenerate
    band group (projection >= 1 - 1e-6).  As a check that the files hold eigenvectors,
    every field of a nonzero frequency satisfies C^H C E = w^2 B E against the oracle's
    sparse curl to a relative residual of 1e-2: the files keep 7 significant digits
    (the reference's "% e" format), and C^H C (norm about 3000 at 16^3) amplifies that
    rounding to residuals of about 1e-4."""
    if not os.path.exists(DROPIN):
        pytest.skip("fame_b200_main not built (needs the reference sources)")
    import fame_oracle as fo
    from fixtures import edge_eps, load_pre
    par = load_pre("sc16")
    B = edge_eps(par)
    build, nx, pn, eps_in, eps_out, nw, ns = ri.WORKLOADS["sc16"]
    runs = {}
    for tag, env in (("batched", None), ("single", {"FAME_B200_SAVE_BATCH": "1"})):
        d = str(tmp_path / tag)
        ri.write_workdir(d, "Syn_sc16", build(), nx, pn, eps_in, eps_out, nw, ns, 1e-10, 100, 1e-10, 1000,
                         flags=(0, 0, 0, 0, 0, 1))
        r = _run(DROPIN, d, env)
        assert r.returncode == 0, r.stderr[-2000:]
        runs[tag] = (d, np.abs(_read_omega(os.path.join(d, "Data_Omega_array.txt"))))
    (db, wb), (ds, ws) = runs["batched"], runs["single"]
    nk = wb.shape[0]
    assert nk >= 2 and nk == len(par["kpoints"])
    assert np.max(np.abs(wb - ws) / np.maximum(ws, 1e-300)) < 1e-10
    names = sorted(n for n in os.listdir(db) if n.startswith("Data_EV_"))
    assert names == sorted(n for n in os.listdir(ds) if n.startswith("Data_EV_"))
    assert len(names) == nk * nw
    ev = lambda d, q, b: _read_ev(os.path.join(d, f"Data_EV_{q + 1:02d}_{b + 1:02d}.txt"))
    for q in range(nk):
        live = [b for b in range(nw) if wb[q, b] > 0]  # the Gamma point's two zero bands aside
        Eb = {b: ev(db, q, b) for b in live}
        Es = {b: ev(ds, q, b) for b in live}
        for b in live:
            assert Eb[b].size == 3 * par["N"]
            assert fo.relative_residual_simple(Eb[b], wb[q, b], par["kpoints"][q], par, B) < 1e-2
            group = [c for c in live if abs(wb[q, c] - wb[q, b]) <= 1e-6 * wb[q, b]]
            Q, _ = np.linalg.qr(np.stack([Es[c] for c in group], axis=1))
            v = Eb[b] / np.linalg.norm(Eb[b])
            assert np.linalg.norm(Q.conj().T @ v) > 1 - 1e-6
