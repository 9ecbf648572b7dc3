"""The oracle's Brent root finder (stand-in for GSL's, which the reference links)."""
import ctypes
import math
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class Brent(ctypes.Structure):
    _fields_ = [("f", ctypes.c_void_p), ("params", ctypes.c_void_p)] + \
               [(n, ctypes.c_double) for n in ("a", "b", "c", "fa", "fb", "fc", "d", "e", "lower", "upper")]


FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double, ctypes.c_void_p)


@pytest.mark.parametrize("f,lo,hi,root", [
    (lambda x, p: x * x - 2.0, 0.0, 2.0, math.sqrt(2.0)),
    (lambda x, p: math.cos(x) - x, 0.0, 1.0, 0.7390851332151607),
    (lambda x, p: (x - 1e-7) * 1e3, 0.0, 1.0, 1e-7),
])
def test_brent_converges(f, lo, hi, root):
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    cb = FN(f)
    s = Brent()
    lib.oracle_brent_set.argtypes = [ctypes.POINTER(Brent), FN, ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
    assert lib.oracle_brent_set(ctypes.byref(s), cb, None, lo, hi) == 0
    lib.oracle_brent_iterate.argtypes = [ctypes.POINTER(Brent)]
    lib.oracle_brent_continue.argtypes = [ctypes.c_double] * 4
    for _ in range(200):
        lib.oracle_brent_iterate(ctypes.byref(s))
        if not lib.oracle_brent_continue(s.lower, s.upper, 0.0, 1e-13):
            break
    assert abs(s.b - root) <= 1e-12 * abs(root)
