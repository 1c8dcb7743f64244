"""Eigenvector text files (fame_write_eigenvectors, fame_writer_start/finish) on the
CPU: byte for byte the reference's FAME_Save_Eigenvector
(FAME_Tools/FAME_Save_Eigenvector.cpp:7-45, built from its source into
oracle/_ref/fame_ref_evwriter by oracle/build_ref.sh; skipped where absent), the
same bytes from one thread and from many, the values read back within the 7
significant digits of "% e", and the error paths."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import fame_b200 as fb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EVW = os.path.join(ROOT, "oracle", "_ref", "fame_ref_evwriter")


def _vectors(nwant, n3, seed=3):
    rng = np.random.default_rng(seed)
    v = (rng.standard_normal((nwant, n3)) * 10.0 ** rng.integers(-12, 12, (nwant, n3))
         + 1j * rng.standard_normal((nwant, n3)))
    special = [0.0, -0.0, 5e-324, -2.5e-310, 1.7976931348623157e308, np.inf, -np.inf, np.nan, 0.5, 9.9999995e-7,
               1.0000005, -123456.75]
    v.real[0, :len(special)] = special
    v.imag[-1, :len(special)] = special[::-1]
    return v


def _files(d, kidx, nwant):
    return [os.path.join(d, f"Data_EV_{kidx + 1:02d}_{b + 1:02d}.txt") for b in range(nwant)]


def _read(path):
    with open(path, "rb") as f:
        return f.read()


def test_threads_write_the_same_bytes_and_values_read_back(tmp_path):
    nwant, n3, kidx = 3, 200003, 11
    v = _vectors(nwant, n3)
    d1, d8 = tmp_path / "t1", tmp_path / "t8"
    d1.mkdir()
    d8.mkdir()
    fb.write_eigenvectors(v, kidx, str(d1), nthreads=1)
    fb.write_eigenvectors(v, kidx, str(d8), nthreads=8)
    for a, b in zip(_files(str(d1), kidx, nwant), _files(str(d8), kidx, nwant)):
        assert _read(a) == _read(b)
    lines = _read(_files(str(d1), kidx, nwant)[0]).decode().splitlines()
    assert lines[0] == "Ele_field_mtx{12}(:, 1) = [" and lines[-1] == "];"
    assert len(lines) == n3 + 2
    pat = re.compile(r"^\((.+)\) \+ \((.+) \* 1i\)$")
    parts = [pat.match(l).groups() for l in lines[1:-1]]
    re_, im_ = np.array([float(a) for a, _ in parts]), np.array([float(b) for _, b in parts])
    for got, want in ((re_, v[0].real), (im_, v[0].imag)):
        assert np.array_equal(np.isnan(got), np.isnan(want))
        ok = ~np.isnan(want)
        assert np.allclose(got[ok], want[ok], rtol=6e-7, atol=0)


@pytest.mark.skipif(not os.path.exists(REF_EVW), reason="oracle/_ref/fame_ref_evwriter not built")
@pytest.mark.parametrize("kidx,nwant", [(0, 2), (9, 3), (99, 1)])
def test_bytes_match_the_reference_writer(tmp_path, kidx, nwant):
    n3 = 5003
    v = _vectors(nwant, n3, seed=kidx)
    ref, ours = tmp_path / "ref", tmp_path / "ours"
    ref.mkdir()
    ours.mkdir()
    inp = tmp_path / "in.bin"
    v.astype("<c16").tofile(inp)
    subprocess.run([REF_EVW, str(nwant), str(n3), str(kidx), str(inp)], cwd=ref, check=True)
    w = C.c_void_p()
    lib = fb.load()
    ev = np.ascontiguousarray(v)
    assert lib.fame_writer_start(os.fsencode(str(ours)), ev.ctypes.data_as(C.POINTER(C.c_double)), nwant, n3,
                                 kidx, 4, C.byref(w)) == fb.OK
    assert lib.fame_writer_finish(w) == fb.OK
    names = sorted(os.listdir(ref))
    assert names == sorted(os.listdir(ours)) == sorted(os.path.basename(p) for p in _files(".", kidx, nwant))
    for n in names:
        assert _read(ref / n) == _read(ours / n), n


def test_errors_are_reported(tmp_path):
    lib = fb.load()
    v = np.zeros((1, 4), np.complex128)
    p = v.ctypes.data_as(C.POINTER(C.c_double))
    assert lib.fame_write_eigenvectors(None, None, 1, 4, 0, 1) == fb.ERR_BAD_INPUT
    assert lib.fame_write_eigenvectors(None, p, 0, 4, 0, 1) == fb.ERR_BAD_INPUT
    missing = os.fsencode(str(tmp_path / "no" / "such" / "dir"))
    assert lib.fame_write_eigenvectors(missing, p, 1, 4, 0, 1) == fb.ERR_IO
    assert "cannot open" in lib.fame_last_error().decode()
    w = C.c_void_p()
    assert lib.fame_writer_start(missing, p, 1, 4, 0, 1, C.byref(w)) == fb.OK
    assert lib.fame_writer_finish(w) == fb.ERR_IO
    assert "cannot open" in lib.fame_last_error().decode()
    assert lib.fame_writer_finish(None) == fb.ERR_BAD_INPUT


def test_default_directory_is_the_working_directory(tmp_path, monkeypatch):
    """dir = NULL writes into the working directory, as the reference's writer does;
    two background writers run at once into different directories."""
    monkeypatch.chdir(tmp_path)
    v = _vectors(2, 1001, seed=5)
    fb.write_eigenvectors(v, 4)
    assert sorted(os.listdir(tmp_path)) == ["Data_EV_05_01.txt", "Data_EV_05_02.txt"]
    lib = fb.load()
    ev = np.ascontiguousarray(v)
    ws = []
    for d in ("a", "b"):
        (tmp_path / d).mkdir()
        w = C.c_void_p()
        assert lib.fame_writer_start(os.fsencode(str(tmp_path / d)), ev.ctypes.data_as(C.POINTER(C.c_double)), 2,
                                     1001, 4, 2, C.byref(w)) == fb.OK
        ws.append(w)
    for w in ws:
        assert lib.fame_writer_finish(w) == fb.OK
    for n in ("Data_EV_05_01.txt", "Data_EV_05_02.txt"):
        assert _read(tmp_path / n) == _read(tmp_path / "a" / n) == _read(tmp_path / "b" / n)
