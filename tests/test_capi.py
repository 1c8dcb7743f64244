"""The C ABI library loads, exports exactly what include/fame_b200.h declares, and
fails loudly (status codes, no fallback) where no device is present."""
import ctypes as C
import os
import re

import pytest

import fame_b200 as fb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fame_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fame_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_python_export_list():
    assert declared_functions() == sorted(fb.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = fb.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert fb.version().startswith("fame-b200")


def test_null_arguments_are_rejected():
    lib = fb.load()
    assert lib.fame_ctx_create(0, None, None) == fb.ERR_BAD_INPUT
    assert lib.fame_set_eps(None, None) == fb.ERR_BAD_INPUT
    assert lib.fame_solve_kpoints(None, None, 0, None, None, None, None, None, None, None) == fb.ERR_BAD_INPUT
    assert b"null" in lib.fame_last_error()


def test_struct_layouts_match_header():
    # fame_lattice: 3 int + 3 double + 9 double + int + 4 int + 3 double
    assert C.sizeof(fb.Lattice) == 4 * 3 + 4 + 8 * 3 + 8 * 9 + 4 + 4 * 4 + 4 + 8 * 3
    assert C.sizeof(fb.KCounters) == 7 * 4


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and
                    __import__("torch").cuda.is_available(), reason="a GPU is visible")
def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(fb.FameError) as e:
        fb.Context((8, 8, 8), [1 / 8] * 3, [1, 0, 0, 0, 1, 0, 0, 0, 1], True)
    assert e.value.code == fb.ERR_NO_DEVICE


def test_reduced_size_follows_the_gamma_rule():
    simple = fb.make_lattice((4, 4, 4), [0.25] * 3, [1, 0, 0, 0, 1, 0, 0, 0, 1], True)
    general = fb.make_lattice((4, 4, 4), [0.25] * 3, [1, 0, 0, 0, 1, 0, 0, 0, 1], False)
    assert fb.reduced_size(simple, [0, 0, 0]) == 63
    assert fb.reduced_size(simple, [5e-5, 0, 0]) == 63
    assert fb.reduced_size(simple, [5e-4, 0, 0]) == 64
    assert fb.reduced_size(general, [5e-4, 0, 0]) == 63
    assert fb.reduced_size(general, [2e-3, 0, 0]) == 64
    with pytest.raises(ValueError):
        fb.reduced_size(simple, [0, 0])


def test_qbq_static_rejects_tensors_before_any_device_call():
    """Host tensors, wrong dtypes and wrong sizes raise ValueError in the wrapper: the
    library would read and write 2*Nd (3N) elements at the raw pointers."""
    torch = pytest.importorskip("torch")
    lat = fb.make_lattice((4, 4, 4), [0.25] * 3, [1, 0, 0, 0, 1, 0, 0, 0, 1], True)
    k = [0.1, 0.0, 0.0]
    x = torch.zeros(128, dtype=torch.complex128)
    inv_b = torch.ones(192, dtype=torch.float64)
    with pytest.raises(ValueError, match="CUDA"):
        fb.qbq_static(lat, k, inv_b, x, x)
    with pytest.raises(ValueError, match="torch tensor"):
        fb.qbq_static(lat, k, inv_b.numpy(), x, x)
