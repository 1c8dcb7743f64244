"""fame_material_locate (the material index map Binout on the GPU) against the
reference's own CPU FAME_Material_Locate_Index output, bit-exact, for every
preprocessed workload in tests/golden/*_pre.npz (simple cubic, FCC, BCC and
hexagonal lattices, spheres and cylinders, one to four materials, grids up to
128x107x92)."""
import numpy as np
import pytest

import fame_b200 as fb
from fixtures import load_pre

pytestmark = pytest.mark.gpu

NAMES = ["sc16", "sc32", "sc96", "fcc16", "fcc64", "bcc12", "bcc48", "hex12", "hex128"]


@pytest.mark.parametrize("name", NAMES)
def test_binout_bit_exact(name):
    par = load_pre(name)
    b = fb.material_locate(par["grid"], par["mesh_len"], par["lattice_vec_a"], par["Omega"], par["Permutation"],
                           par["material"])
    assert b.shape == par["binout"].shape
    assert np.array_equal(b, par["binout"]), int(np.sum(b != par["binout"]))
