"""Device arithmetic helpers of physics.cuh that replace a library call or a
plain divide and must give the same bits, run on the GPU through the test
suite's self-test library (gamma_b200/lib/libgamma_selftest.so):

- gb::pow_3_4, the isentrope x^(3/4) of the shock detector: x^0.75 rounded to
  nearest, as the C library's pow returns it to the reference (1/GAMMA_ = 0.75
  exactly for GAMMA_ = 4/3).  The correctly rounded value is computed here with
  60-digit decimal arithmetic; CUDA's own pow is evaluated beside it for
  comparison only.
- gb::qdiv, the quotient that keeps zero numerators away from the divide's
  slow path: the IEEE quotient bit for bit.
"""
import ctypes
import decimal
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gamma_b200", "lib",
                   "libgamma_selftest.so")


def _correctly_rounded(x):
    decimal.getcontext().prec = 60
    e = decimal.Decimal("0.75")
    return np.array([float(decimal.Decimal(float(v)) ** e) for v in x])


def test_pow_3_4_is_correctly_rounded(gpu_available):
    assert os.path.exists(LIB), "build the self-test library: make -C gamma_b200/csrc"
    lib = ctypes.CDLL(LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.gb_selftest_pow_3_4.argtypes = [dp, dp, dp, ctypes.c_int]
    rng = np.random.default_rng(7)
    x = np.concatenate([
        np.exp(rng.uniform(np.log(1e-12), 0., 20000)),       # p/p1 of the detector's integral
        1. - rng.uniform(0., 1e-6, 4000),                     # weak pressure jumps
        np.exp(rng.uniform(np.log(1e-270), np.log(1e270), 6000)),
        np.array([1., 0.5, 0.25, 2.0 ** -800, 2.0 ** 800, 2.0 ** -900, 2.0 ** 900]),
    ])
    edge = np.array([0.0, 2.0 ** -1000, 1e300, np.inf, np.nan, -1.0])  # outside [2^-900, 2^900]: pow itself
    x = np.concatenate([x, edge])
    n_edge = edge.size
    mine, libm = np.zeros_like(x), np.zeros_like(x)
    rc = lib.gb_selftest_pow_3_4(x.ctypes.data_as(dp), mine.ctypes.data_as(dp), libm.ctypes.data_as(dp), x.size)
    assert rc == 0
    main = slice(0, x.size - n_edge)
    cr = _correctly_rounded(x[main])
    bad = np.flatnonzero(mine[main] != cr)
    assert bad.size == 0, (bad.size, x[bad[:5]], mine[bad[:5]], cr[bad[:5]])
    assert np.array_equal(mine[main.stop:], libm[main.stop:], equal_nan=True)
    # CUDA's pow (documented to 2 ulp) is the comparison point, not a requirement
    assert np.all(np.abs(libm[main] - cr) <= 2 * np.spacing(cr))


def test_qdiv_is_the_ieee_quotient(gpu_available):
    """gb::qdiv (zero numerators kept away from the divide's slow path) returns
    a / b bit for bit: signed zeros, infinities, NaN, subnormals, and ordinary
    pairs."""
    lib = ctypes.CDLL(LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.gb_selftest_qdiv.argtypes = [dp, dp, dp, dp, ctypes.c_int]
    special = np.array([0.0, -0.0, 1.0, -1.0, 5e-324, -5e-324, 2.2250738585072014e-308, 1e-310, 1e300, -1e300,
                        np.inf, -np.inf, np.nan])
    a = np.repeat(special, special.size)
    b = np.tile(special, special.size)
    rng = np.random.default_rng(3)
    ra = rng.standard_normal(20000) * np.exp(rng.uniform(-300, 300, 20000))
    rb = rng.standard_normal(20000) * np.exp(rng.uniform(-300, 300, 20000))
    ra[::3] = 0.0
    ra[1::7] = -0.0
    a = np.concatenate([a, ra])
    b = np.concatenate([b, rb])
    mine, ieee = np.zeros_like(a), np.zeros_like(a)
    rc = lib.gb_selftest_qdiv(a.ctypes.data_as(dp), b.ctypes.data_as(dp), mine.ctypes.data_as(dp),
                              ieee.ctypes.data_as(dp), a.size)
    assert rc == 0
    same = (mine.view(np.uint64) == ieee.view(np.uint64)) | (np.isnan(mine) & np.isnan(ieee))
    bad = np.flatnonzero(~same)
    assert bad.size == 0, (a[bad[:5]], b[bad[:5]], mine[bad[:5]], ieee[bad[:5]])
    with np.errstate(all="ignore"):
        host = a / b  # the host's IEEE quotient too
    same_host = (mine.view(np.uint64) == host.view(np.uint64)) | (np.isnan(mine) & np.isnan(host))
    assert np.all(same_host)
