"""ctypes access to the compiled GAMMA reference (oracle/_ref/libref_*.so).

TEST INFRASTRUCTURE.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg use this module, as the checker or as the timed CPU reference.

Each library holds one process-wide ``Simu`` (the reference keeps its grid in
globals and file statics), so a fresh configuration needs a fresh process when
parameters of the problem module change; :func:`run_isolated` does that with a
``spawn`` pool.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


@dataclass
class Snapshot:
    """One track: cells [0, ntrack), interfaces [0, ntrack-1)."""

    t: float
    dt: float
    it: int
    ntrack: int
    prim: np.ndarray  # [NQ, ntrack]
    x: np.ndarray
    dx: np.ndarray
    dt_loc: np.ndarray
    sd: np.ndarray
    pspec: np.ndarray
    shocked: np.ndarray
    xI: np.ndarray  # [ntrack-1]

    @property
    def ngst(self) -> int:
        return 2


class RefSim:
    """One reference build (``kind`` in {bm1d, bm1d_orig, tube, bm1d_synge,
    bm1d_euler, tube_euler (Timestep/euler.cpp in place of rk3.cpp)}, or
    bm1d_io / tube_io: the reference's own text IO module linked, so printCols
    writes ../results/Last/phys*.out relative to the working directory and
    resume() reads the last one back)."""

    def __init__(self, kind: str):
        path = os.path.join(REF_DIR, f"libref_{kind}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        self.kind = kind
        lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
        lib.ref_nq.restype = ctypes.c_int
        lib.ref_gamma_ad.restype = ctypes.c_double
        lib.ref_init.restype = ctypes.c_int
        lib.ref_step.argtypes = [ctypes.c_int]
        lib.ref_snapshot.restype = ctypes.c_int
        lib.ref_snapshot.argtypes = [_dp] * 8 + [ctypes.c_int]
        lib.ref_scalars.argtypes = [_dp]
        lib.ref_load.argtypes = [ctypes.c_int] + [_dp] * 5 + [ctypes.c_int, ctypes.c_double, ctypes.c_long]
        lib.ref_cons2prim.argtypes = [_dp, _dp, _dp, ctypes.c_int]
        lib.ref_prim2cons.argtypes = [_dp, _dp, _dp, ctypes.c_int]
        lib.ref_riemann.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
        if hasattr(lib, "ref_set_param"):
            lib.ref_set_param.argtypes = [ctypes.c_char_p, ctypes.c_double]
            lib.ref_set_param.restype = ctypes.c_int
        if hasattr(lib, "ref_set_c2p_epsrel"):
            lib.ref_set_c2p_epsrel.argtypes = [ctypes.c_double]
        lib.ref_resume.restype = ctypes.c_int
        if hasattr(lib, "ref_bm1d_derived"):
            lib.ref_bm1d_derived.argtypes = [_dp]
        self.lib = lib
        self.nq = lib.ref_nq()
        self.gamma_ad = lib.ref_gamma_ad()
        self.shock_detection = bool(lib.ref_shock_detection())
        self.synchrotron = bool(lib.ref_local_synchrotron())

    # -- set-up -----------------------------------------------------------------
    def set_params(self, **params):
        for k, v in params.items():
            if self.lib.ref_set_param(k.encode(), float(v)) != 0:
                raise KeyError(f"unknown parameter {k} for {self.kind}")

    def init(self):
        self.lib.ref_init()

    def print_cols(self):
        """Grid::printCols at the current iteration (io builds write a file)."""
        self.lib.ref_print_cols()

    def resume(self):
        """main.cpp's -r start from the last ../results/Last/phys*.out (io builds)."""
        if self.lib.ref_resume() != 0:
            raise FileNotFoundError("../results/Last missing")

    def set_c2p_epsrel(self, epsrel: float):
        """cons2prim's Brent stopping tolerance (1e-13 in the reference; 0 restores it)"""
        self.lib.ref_set_c2p_epsrel(float(epsrel))

    def bm1d_derived(self) -> dict:
        out = np.zeros(8)
        self.lib.ref_bm1d_derived(_ptr(out))
        keys = ["tstart", "RShock", "lfacShock2", "rhoNorm", "pNorm", "lNorm", "vNorm"]
        return dict(zip(keys, out.tolist()))

    # -- stepping ---------------------------------------------------------------
    def step(self, n: int = 1):
        self.lib.ref_step(int(n))

    def regrid(self):
        self.lib.ref_regrid()

    def scalars(self) -> dict:
        out = np.zeros(8)
        self.lib.ref_scalars(_ptr(out))
        keys = ["t", "dt", "it", "ntrack", "nact", "iLbnd", "iRbnd", "cap"]
        return dict(zip(keys, out.tolist()))

    def snapshot(self) -> Snapshot:
        sc = self.scalars()
        cap = int(sc["cap"])
        prim = np.zeros((self.nq, cap))
        arrs = [np.zeros(cap) for _ in range(6)]
        xI = np.zeros(cap)
        n = self.lib.ref_snapshot(_ptr(prim), *[_ptr(a) for a in arrs], _ptr(xI), cap)
        assert n >= 0
        return Snapshot(
            t=sc["t"], dt=sc["dt"], it=int(sc["it"]), ntrack=n,
            prim=prim[:, :n].copy(), x=arrs[0][:n].copy(), dx=arrs[1][:n].copy(),
            dt_loc=arrs[2][:n].copy(), sd=arrs[3][:n].copy(), pspec=arrs[4][:n].copy(),
            shocked=arrs[5][:n].copy(), xI=xI[: n - 1].copy(),
        )

    def load(self, snap: Snapshot):
        n = snap.ntrack
        cap = n
        prim = np.ascontiguousarray(snap.prim[:, :n], dtype=np.float64)
        rc = self.lib.ref_load(
            n, _ptr(prim), _ptr(np.ascontiguousarray(snap.x)), _ptr(np.ascontiguousarray(snap.dx)),
            _ptr(np.ascontiguousarray(snap.dt_loc)), _ptr(np.ascontiguousarray(snap.xI)), cap,
            float(snap.t), int(snap.it))
        if rc != 0:
            raise ValueError("track does not fit the reference grid capacity")

    # -- per-state kernels --------------------------------------------------------
    def cons2prim(self, cons: np.ndarray, prim_guess: np.ndarray, r=None):
        cons = np.ascontiguousarray(cons, dtype=np.float64).copy()
        prim = np.ascontiguousarray(prim_guess, dtype=np.float64).copy()
        n = cons.shape[1]
        rr = None if r is None else np.ascontiguousarray(r, dtype=np.float64)
        self.lib.ref_cons2prim(_ptr(cons), _ptr(prim), _ptr(rr), n)
        return prim, cons

    def prim2cons(self, prim: np.ndarray, r=None):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        cons = np.zeros_like(prim)
        rr = None if r is None else np.ascontiguousarray(r, dtype=np.float64)
        self.lib.ref_prim2cons(_ptr(prim), _ptr(cons), _ptr(rr), prim.shape[1])
        return cons

    def riemann(self, primL, primR, x, v=None):
        primL = np.ascontiguousarray(primL, dtype=np.float64)
        primR = np.ascontiguousarray(primR, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = primL.shape[1]
        vv = np.zeros(n) if v is None else np.ascontiguousarray(v, dtype=np.float64)
        lam = np.zeros(3 * n)
        flux = np.zeros((self.nq, n))
        self.lib.ref_riemann(_ptr(primL), _ptr(primR), _ptr(x), _ptr(vv), 0 if v is None else 1,
                             _ptr(lam), _ptr(flux), n)
        return lam.reshape(n, 3), flux


def _worker(args):
    kind, params, nsteps, snap_at, epsrel = args
    sim = RefSim(kind)
    sim.set_params(**params)
    sim.init()
    if epsrel:
        sim.set_c2p_epsrel(epsrel)
    out = {0: sim.snapshot()} if 0 in snap_at else {}
    done = 0
    for s in sorted(x for x in snap_at if x > 0):
        sim.step(s - done)
        done = s
        out[s] = sim.snapshot()
    if nsteps > done:
        sim.step(nsteps - done)
    return out


def run_isolated(kind: str, params: dict, nsteps: int, snap_at=(0,), c2p_epsrel: float = 0.):
    """Run one configuration in a fresh spawned process; returns {step: Snapshot}.
    c2p_epsrel > 0 replaces the reference's cons2prim stopping tolerance after
    the initial state is built."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply(_worker, ((kind, params, nsteps, tuple(snap_at), c2p_epsrel),))
