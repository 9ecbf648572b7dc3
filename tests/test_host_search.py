"""The 2D passes' search from a hint (`partition_from`, gamma_b200/csrc/
search.cuh) against a linear scan, run on the host through the test suite's
self-test library (gamma_b200/lib/libgamma_selftest.so).

The neighbour lists (the first interface of the adjacent track at or above a
cell's lower edge, computeNeighbors in 2d.cpp) and the theta gather (the
lower-track cells whose upper lists hold a cell) search from hints left in
memory by the previous stage or by the cell's own list; the GPU results are
bit-identical to a plain binary search only if the search returns the
binary search's index for every hint, including hints far out of range.
"""
import ctypes
import os

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gamma_b200", "lib",
                   "libgamma_selftest.so")


def test_partition_from_matches_linear_scan():
    assert os.path.exists(LIB), "build the self-test library: make -C gamma_b200/csrc"
    lib = ctypes.CDLL(LIB)
    lib.gb_selftest_partition_from.argtypes = [ctypes.c_uint, ctypes.c_int]
    lib.gb_selftest_partition_from.restype = ctypes.c_int
    # random sorted arrays of 0-40 entries with ties, keys around their range,
    # hints in range and up to 1e6 outside it; -1 would mean a probe left the
    # range (an out-of-bounds load on the GPU)
    for seed in (7, 12345, 2024):
        assert lib.gb_selftest_partition_from(seed, 200000) == 0, seed
