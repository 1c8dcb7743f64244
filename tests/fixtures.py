"""Loaders for the committed golden fixtures in tests/golden/ (test helpers)."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_pre(name):
    """Reference preprocessing output for a named workload as a dict."""
    z = np.load(os.path.join(GOLDEN, f"{name}_pre.npz"))
    n = int(z["Binout_len"])
    binout = np.unpackbits(z["Binout_bits"])[:n].astype(np.int32)
    grid = tuple(int(v) for v in z["grid_nums"])
    par = dict(
        name=name,
        grid=grid,
        N=int(np.prod(grid)),
        mesh_len=z["mesh_len"].astype(float),
        edge_len=z["edge_len"].astype(float),
        lattice_vec_a=z["lattice_vec_a"].astype(float),
        lattice_vec_a_orig=z["lattice_vec_a_orig"].astype(float),
        Omega=z["Omega"].astype(float),
        Permutation=[int(v) for v in z["Permutation"]],
        m=tuple(int(v) for v in z["m"]),
        t=z["t"].astype(float),
        t1=z["t"][:3].astype(float),
        simple=bool(int(z["simple"][0])),
        material_num=int(z["material_num"][0]),
        binout=binout,
        eps_in=[float(v) for v in z["ele_permitt_in"]],
        eps_out=float(z["ele_permitt_out"][0]),
        kpoints=z["WaveVector"].reshape(-1, 3).astype(float),
        material=json.loads(str(z["material"])),
    )
    return par


def edge_eps(par):
    """B (3N) with FAME_Matrix_B_Isotropic's last-material-wins rule."""
    import fame_oracle as fo
    return fo.matrix_B(par["binout"], par["material_num"], par["eps_in"], par["eps_out"], par["N"])


def load_ref(name):
    with open(os.path.join(GOLDEN, f"{name}_ref.json")) as f:
        return json.load(f)


def load_apply(name):
    return np.load(os.path.join(GOLDEN, f"{name}_apply.npz"))


def lattice_struct(par):
    """Fields of the C ABI fame_lattice for a workload."""
    return dict(grid=par["grid"], mesh_len=list(par["mesh_len"]), lattice_vec_a=list(par["lattice_vec_a"]),
                simple=int(par["simple"]), m=list(par["m"]), t1=list(par["t1"]))
