"""Input files for the reference build in oracle/_ref (test infrastructure only).

Writes a work directory the reference's Main.out / fame_ref_harness accept:
Popt.txt in the format FAME_Preprocessing/FAME_Set_User_Option.cpp:13-140 parses,
and FAME_Material_Data/<name>.txt in the format of
FAME_Preprocessing/FAME_Set_User_Define.cpp:24-121.  Also parses the binary dump
written by `fame_ref_harness pre`.

The named configurations are the band-structure workloads used across tests and
bench.py; their material descriptions are synthetic (no dataset is involved).
"""
from __future__ import annotations

import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_HARNESS = os.path.join(HERE, "_ref", "fame_ref_harness")


def material(lattice_type, const, spheres=(), cylinders=(), material_num=1):
    """spheres: list of (kind, (cx,cy,cz), r); cylinders: (kind, top, bot, r).
    Centres are fractional coordinates in the lattice vectors."""
    return dict(lattice_type=lattice_type, const=tuple(const), spheres=list(spheres),
                cylinders=list(cylinders), material_num=material_num)


def _fmt(v):
    return " ".join(f"{float(x):.12f}" for x in v)


def write_workdir(path, name, mat, grid_nx, part_num, eps_in, eps_out, nwant, nstep,
                  es_tol, es_maxit, ls_tol, ls_maxit, flags=(0, 0, 0, 0, 0, 0)):
    os.makedirs(os.path.join(path, "FAME_Material_Data"), exist_ok=True)
    nm = mat["material_num"]
    sph = [[s for s in mat["spheres"] if s[0] == k] for k in range(nm)]
    cyl = [[c for c in mat["cylinders"] if c[0] == k] for k in range(nm)]
    lines = ["# Data name", f" {name}", "# Material number", f" {nm}", "# Lattice type",
             f" {mat['lattice_type']}", "# Lattice constant", " " + _fmt(mat["const"]),
             "# Sphere number"]
    lines += [f" {len(s)}" for s in sph]
    lines += ["# Sphere centers"]
    lines += [" " + _fmt(s[1]) for k in range(nm) for s in sph[k]]
    lines += ["# Sphere radius"]
    lines += [" " + _fmt([s[2]]) for k in range(nm) for s in sph[k]]
    lines += ["# Cylinder number"]
    lines += [f" {len(c)}" for c in cyl]
    lines += ["# Cylinder top centers"]
    lines += [" " + _fmt(c[1]) for k in range(nm) for c in cyl[k]]
    lines += ["# Cylinder bot centers"]
    lines += [" " + _fmt(c[2]) for k in range(nm) for c in cyl[k]]
    lines += ["# Cylinder radius"]
    lines += [" " + _fmt([c[3]]) for k in range(nm) for c in cyl[k]]
    with open(os.path.join(path, "FAME_Material_Data", name + ".txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    pr_user, pr_par, cr_par, cr_b, cr_wv, save_ev = flags
    popt = [
        "# Grid number", f" {grid_nx} {grid_nx} {grid_nx}", "",
        "# Part number", f" {part_num}", "",
        "# Material data name", f" {name}",
        "# Material type", " isotropic",
        "# Permittivity (inner material)", f" {len(eps_in)}", " " + " ".join(repr(float(e)) for e in eps_in),
        "# Permittivity (outer material)", f" {float(eps_out)!r}", "",
        "# Desired eigenpair number", f" {nwant}",
        "# Dimension of Krylov subspace for Lanczos", f" {nstep}",
        "# Tolerance of Lanczos", f" {es_tol:.6e}",
        "# Maximum restart number of Lanczos", f" {es_maxit}",
        "# Tolerance of linear solver", f" {ls_tol:.6e}",
        "# Maximum iteration number of linear solver", f" {ls_maxit}", "",
        "# Device", " 0",
        "# Printf User Option", f" {pr_user}",
        "# Printf Parameter", f" {pr_par}",
        "# Create Parameter", f" {cr_par}",
        "# Create B_inout", f" {cr_b}",
        "# Create Wave Vector", f" {cr_wv}",
        "# Save Eigen Vector", f" {save_ev}",
        "# Grid nums Max", " 0 16",
        "# Sphere/Cylinder radius adjustment", " 0 0.6",
    ]
    with open(os.path.join(path, "Popt.txt"), "w") as f:
        f.write("\n".join(popt) + "\n")


def parse_pre(path):
    """Parse the record stream written by fame_ref_harness `pre` (oracle/ref_harness.cu)."""
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    p = 0
    while p < len(data):
        (ln,) = struct.unpack_from("<i", data, p)
        p += 4
        name = data[p:p + ln].decode()
        p += ln
        dt = chr(data[p])
        p += 1
        (n,) = struct.unpack_from("<q", data, p)
        p += 8
        w = 4 if dt == "i" else 8
        arr = np.frombuffer(data, dtype="<i4" if dt == "i" else "<f8", count=n, offset=p).copy()
        p += n * w
        out[name] = arr
    return out


def run_pre(workdir, out_bin):
    subprocess.run([REF_HARNESS, "pre", workdir, out_bin], check=True,
                   stdout=subprocess.DEVNULL)
    return parse_pre(out_bin)


# ---------------------------------------------------------------- named workloads
def _sc_sphere():
    return material("simple_cubic", (1, 0, 0, 0, 0, 0), spheres=[(0, (0, 0, 0), 0.25)])


def _fcc_two_spheres():
    return material("face_centered_cubic", (1, 0, 0, 0, 0, 0),
                    spheres=[(0, (0, 0, 0), 0.2), (0, (0.25, 0.25, 0.25), 0.2)])


def _bcc_rods():
    tops = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)]
    return material("body_centered_cubic", (1, 0, 0, 0, 0, 0),
                    cylinders=[(k, tops[k], (0, 0, 0), 0.12) for k in range(4)], material_num=4)


def _hex_honeycomb():
    return material("hexagonal", (1, 0, 1.2, 0, 0, 0),
                    cylinders=[(0, (1 / 3, 2 / 3, 1), (1 / 3, 2 / 3, 0), 0.3),
                               (0, (2 / 3, 1 / 3, 1), (2 / 3, 1 / 3, 0), 0.3)])


def bcc_eps(seed=0):
    return list(np.random.default_rng(seed).uniform(8.0, 14.0, 4))


# name -> (material builder, Popt Nx, part_num, eps_in, eps_out, nwant, nstep)
WORKLOADS = {
    "sc16": (_sc_sphere, 16, 4, [13.0], 1.0, 10, 40),
    "sc32": (_sc_sphere, 32, 4, [13.0], 1.0, 8, 40),
    "sc96": (_sc_sphere, 96, 4, [13.0], 1.0, 10, 40),
    "fcc16": (_fcc_two_spheres, 16, 2, [12.0], 1.0, 10, 40),
    "fcc64": (_fcc_two_spheres, 64, 2, [12.0], 1.0, 10, 40),
    "bcc12": (_bcc_rods, 12, 2, bcc_eps(), 1.0, 12, 40),
    "bcc48": (_bcc_rods, 48, 2, bcc_eps(), 1.0, 12, 40),
    "hex12": (_hex_honeycomb, 12, 2, [11.4], 1.0, 16, 40),
    "hex36": (_hex_honeycomb, 36, 2, [11.4], 1.0, 16, 40),
    "hex128": (_hex_honeycomb, 128, 2, [11.4], 1.0, 16, 40),
}


def make_workdir(name, path, es_tol=1e-10, es_maxit=100, ls_tol=1e-10, ls_maxit=1000,
                 part_num=None, nwant=None, nstep=None):
    build, nx, pn, eps_in, eps_out, nw, ns = WORKLOADS[name]
    write_workdir(path, "Syn_" + name, build(), nx, part_num or pn, eps_in, eps_out,
                  nwant or nw, nstep or ns, es_tol, es_maxit, ls_tol, ls_maxit)
    return path
