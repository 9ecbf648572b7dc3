"""ctypes access to the compiled 2D GAMMA reference (oracle/_ref/libref_jet2d.so).

TEST INFRASTRUCTURE.  Only tests/ and bench.py's CPU arms use this module, as
the checker or as the timed CPU reference.  The library keeps one process-wide
``Simu`` (the reference holds its grid in globals), so each configuration runs
in its own spawned process (:func:`run_isolated`).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_jet2d.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _ptr(a, typ=_dp):
    return a.ctypes.data_as(typ)


@dataclass
class Track:
    """One theta track: cells [0, ntrack), interfaces [0, ntrack-1)."""

    ntrack: int
    nact: int
    iLbnd: int
    iRbnd: int
    prim: np.ndarray     # [NQ, ntrack]
    x: np.ndarray        # r
    dx: np.ndarray       # dr
    th: np.ndarray       # theta of every cell
    dth: np.ndarray
    dt_loc: np.ndarray
    sd: np.ndarray
    pspec: np.ndarray
    shocked: np.ndarray
    grad_mv: np.ndarray  # [NQ, ntrack]
    grad_f1: np.ndarray  # [NQ, ntrack]
    xI: np.ndarray       # [ntrack-1]
    nbr: np.ndarray      # [ntrack, 2 sides, (first flat id, count)]


@dataclass
class Grid2D:
    t: float
    dt: float
    it: int
    cap: int             # cells per track including ghosts (nde_nax[MV])
    jLbnd: int
    jRbnd: int
    tracks: list = field(default_factory=list)


class RefJet2D:
    """io=True loads the build with the reference's own text IO module
    (libref_jet2d_io.so): printCols then writes ../results/Last/phys*.out
    relative to the working directory, and resume() reads it back."""

    def __init__(self, io: bool = False, euler: bool = False, synge: bool = False):
        assert io + euler + synge <= 1
        path = LIB.replace("libref_jet2d.so", "libref_jet2d_io.so") if io else LIB
        if euler:
            path = LIB.replace("libref_jet2d.so", "libref_jet2d_euler.so")
        if synge:  # EOS_ = SYNGE_EOS_, GAMMA_ = 5/3
            path = LIB.replace("libref_jet2d.so", "libref_jet2d_synge.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
        lib.ref_nq.restype = ctypes.c_int
        lib.ref_init.restype = ctypes.c_int
        lib.ref_step.argtypes = [ctypes.c_int]
        lib.ref_scalars.argtypes = [_dp]
        lib.ref_track_info.argtypes = [ctypes.c_int, _ip]
        lib.ref_snapshot.restype = ctypes.c_int
        lib.ref_snapshot.argtypes = [ctypes.c_int] + [_dp] * 12 + [_ip, ctypes.c_int]
        lib.ref_set_param.argtypes = [ctypes.c_char_p, ctypes.c_double]
        lib.ref_set_param.restype = ctypes.c_int
        lib.ref_jet2d_derived.argtypes = [_dp]
        lib.ref_partial.argtypes = [ctypes.c_int]
        lib.ref_set_c2p_epsrel.argtypes = [ctypes.c_double]
        lib.ref_fluxes.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int]
        lib.ref_fluxes.restype = ctypes.c_int
        lib.ref_resume.restype = ctypes.c_int
        self.lib = lib
        self.nq = lib.ref_nq()

    def set_params(self, **params):
        for k, v in params.items():
            if self.lib.ref_set_param(k.encode(), float(v)) != 0:
                raise KeyError(f"unknown parameter {k}")

    def print_cols(self):
        """Grid::printCols at the current iteration (io builds write a file)."""
        self.lib.ref_print_cols()

    def resume(self):
        """main.cpp's -r start from the last ../results/Last/phys*.out (io builds)."""
        if self.lib.ref_resume() != 0:
            raise FileNotFoundError("../results/Last missing")

    def derived(self) -> dict:
        out = np.zeros(8)
        self.lib.ref_jet2d_derived(_ptr(out))
        keys = ["tstart", "RShock", "lfacShock2", "rhoNorm", "pNorm", "lNorm", "vNorm"]
        return dict(zip(keys, out.tolist()))

    def init(self):
        self.lib.ref_init()

    def set_c2p_epsrel(self, epsrel: float):
        """cons2prim's Brent stopping tolerance (1e-13 in the reference; 0 restores it)"""
        self.lib.ref_set_c2p_epsrel(float(epsrel))

    def step(self, n: int = 1):
        self.lib.ref_step(int(n))

    def regrid(self):
        self.lib.ref_regrid()

    def partial(self, what: int):
        """regrid, resetShock, updateGhosts (what=1) and prepForUpdate (what=2)"""
        self.lib.ref_partial(int(what))

    def fluxes(self, j: int, cap: int):
        """(cell fluxes [side, dim, q, i], interface v, lL, lR, flux[q]) of track j"""
        out = np.zeros(2 * 2 * self.nq * cap)
        itf = np.zeros((3 + self.nq) * cap)
        n = self.lib.ref_fluxes(int(j), _ptr(out), _ptr(itf), int(cap))
        return out.reshape(2, 2, self.nq, cap)[..., :n], itf.reshape(3 + self.nq, cap)[:, :n - 1]

    def compute_neighbors(self):
        self.lib.ref_compute_neighbors()

    def snapshot(self) -> Grid2D:
        sc = np.zeros(8)
        self.lib.ref_scalars(_ptr(sc))
        nj, cap = int(sc[3]), int(sc[4])
        g = Grid2D(t=sc[0], dt=sc[1], it=int(sc[2]), cap=cap, jLbnd=int(sc[5]), jRbnd=int(sc[6]))
        info = np.zeros(4, dtype=np.int32)
        for j in range(nj):
            self.lib.ref_track_info(j, _ptr(info, _ip))
            prim = np.zeros((self.nq, cap))
            gmv = np.zeros((self.nq, cap))
            gf1 = np.zeros((self.nq, cap))
            a = [np.zeros(cap) for _ in range(8)]
            xI = np.zeros(cap)
            nbr = np.zeros(4 * cap, dtype=np.int32)
            n = self.lib.ref_snapshot(j, _ptr(prim), *[_ptr(v) for v in a], _ptr(gmv), _ptr(gf1), _ptr(xI),
                                      _ptr(nbr, _ip), cap)
            assert n != -1
            if n == -2:
                raise AssertionError(f"track {j}: a neighbour list is not a run of consecutive cells")
            n = int(info[0])
            g.tracks.append(Track(
                ntrack=n, nact=int(info[1]), iLbnd=int(info[2]), iRbnd=int(info[3]),
                prim=prim[:, :n].copy(), x=a[0][:n].copy(), dx=a[1][:n].copy(), th=a[2][:n].copy(),
                dth=a[3][:n].copy(), dt_loc=a[4][:n].copy(), sd=a[5][:n].copy(), pspec=a[6][:n].copy(),
                shocked=a[7][:n].copy(), grad_mv=gmv[:, :n].copy(), grad_f1=gf1[:, :n].copy(),
                xI=xI[:n - 1].copy(), nbr=nbr[:4 * n].reshape(n, 2, 2).copy()))
        return g


def _worker(args):
    params, snap_at, nsteps, epsrel, euler, synge = args
    sim = RefJet2D(euler=euler, synge=synge)
    sim.set_params(**params)
    sim.init()
    if epsrel:
        sim.set_c2p_epsrel(epsrel)
    out = {}
    done = 0
    for s in sorted(snap_at):
        if s > done:
            sim.step(s - done)
            done = s
        out[s] = sim.snapshot()
    if nsteps > done:
        sim.step(nsteps - done)
    return out


def run_isolated(params: dict, snap_at=(0,), nsteps: int = 0, c2p_epsrel: float = 0., euler: bool = False,
                 synge: bool = False):
    """Run one configuration in a fresh spawned process; returns {step: Grid2D}.
    c2p_epsrel > 0 replaces the reference's cons2prim stopping tolerance after
    the initial state is built.  euler: the build with Timestep/euler.cpp;
    synge: the build with the Synge EOS and GAMMA_ = 5/3."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply(_worker, ((params, tuple(snap_at), nsteps, c2p_epsrel, euler, synge),))
