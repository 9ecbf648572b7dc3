"""The C-ABI library loads and exports every symbol include/gamma_gpu.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

from gamma_b200 import gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gamma_gpu.h")).read()
    return sorted(set(re.findall(r"\b(gamma_(?:gpu|mlp|2d|text[12]d)_\w+)\s*\(", src)))


def test_header_matches_binding_list():
    from gamma_b200 import gpu2d
    assert declared_symbols() == sorted(gpu.EXPORTS + gpu2d.EXPORTS)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(gpu.LIB_PATH):
        pytest.fail(f"{gpu.LIB_PATH} missing: run __graft_entry__.build()")
    lib = ctypes.CDLL(gpu.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_strerror_and_invalid_config_without_device():
    assert gpu.strerror(gpu.GAMMA_ERR_NEG_DT).startswith("negative CFL")
    bad = gpu.config_cart()
    bad.nq = 7  # no such module combination
    h = ctypes.c_void_p()
    caps = (ctypes.c_int * 1)(64)
    rc = gpu.lib().gamma_gpu_create(ctypes.byref(bad), 1, caps, ctypes.byref(h))
    assert rc in (gpu.GAMMA_ERR_INVALID, gpu.GAMMA_ERR_NO_DEVICE)


def test_variant_table_matches_binding():
    """the launch-shape table of the library has the binding's size"""
    from gamma_b200 import gpu
    assert gpu.variant_info(0) == (128, 1)
    assert gpu.variant_info(gpu.N_VARIANTS - 1)[0] > 0
    with pytest.raises(gpu.GammaError):
        gpu.variant_info(gpu.N_VARIANTS)
