"""ctypes access to the C restatement of the 1D step (oracle/liboracle.so).

TEST INFRASTRUCTURE -- the oracle.  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg use it, as the checker or the timed CPU port.
Unlike the compiled reference, any number of independent runs can coexist in
one process.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .refsim import Snapshot

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = ctypes.POINTER(ctypes.c_double)

GEOM_SPHERICAL1D, GEOM_CARTESIAN = 0, 1
HYDRO_REL_SPH, HYDRO_REL_CART = 0, 1
EOS_IDEAL, EOS_SYNGE = 0, 1
PROBLEM_BM1D, PROBLEM_TUBE = 0, 1


class OcConfig(ctypes.Structure):
    """Mirror of ``oc_config`` in gamma_oracle.h (same field order)."""

    _fields_ = (
        [(n, ctypes.c_int) for n in ("geometry", "hydro", "eos", "nq", "shock_detection",
                                     "local_synchrotron", "problem", "ngst", "ncell", "nmax")]
        + [(n, ctypes.c_double) for n in ("gamma_ad", "cfl", "vi",
                                          "n0", "eta", "Etot", "n_ext", "tinit", "lfac_shock2",
                                          "lorentz_mode", "Rscale", "k",
                                          "grid_log", "r_lo", "r_hi", "dth", "target_ar", "split_AR",
                                          "merge_AR", "t_bm_until", "v_in", "v_out",
                                          "xmin", "xmax", "xmid", "rhoL", "pL", "vL", "trL",
                                          "rhoR", "pR", "vR", "trR", "c2p_epsrel")]
        + [("eos_wavespeeds", ctypes.c_int), ("timestep", ctypes.c_int)]
    )


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], a.dtype
    return a.ctypes.data_as(_dp)


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle port`")
        L = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
        L.oc_create.restype = ctypes.c_void_p
        L.oc_create.argtypes = [ctypes.POINTER(OcConfig)]
        L.oc_destroy.argtypes = [ctypes.c_void_p]
        L.oc_init.argtypes = [ctypes.c_void_p]
        L.oc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oc_step.restype = ctypes.c_int
        L.oc_regrid.argtypes = [ctypes.c_void_p]
        L.oc_scalars.argtypes = [ctypes.c_void_p, _dp]
        L.oc_snapshot.argtypes = [ctypes.c_void_p] + [_dp] * 8 + [ctypes.c_int]
        L.oc_snapshot.restype = ctypes.c_int
        L.oc_load.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_dp] * 5 + [ctypes.c_int, ctypes.c_double,
                                                                            ctypes.c_long]
        L.oc_load.restype = ctypes.c_int
        L.oc_cons2prim.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.oc_prim2cons.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_int]
        L.oc_riemann.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
        L.oc_bm_profile.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp]
        L.oc_config_bm1d_defaults.argtypes = [ctypes.POINTER(OcConfig)]
        L.oc_config_tube_defaults.argtypes = [ctypes.POINTER(OcConfig)]
        _LIB = L
    return _LIB


def bm1d_config(**overrides) -> OcConfig:
    c = OcConfig()
    lib().oc_config_bm1d_defaults(ctypes.byref(c))
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


def tube_config(**overrides) -> OcConfig:
    c = OcConfig()
    lib().oc_config_tube_defaults(ctypes.byref(c))
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


class PortSim:
    """One run of the restated step."""

    def __init__(self, cfg: OcConfig):
        self.cfg = cfg
        self.nq = cfg.nq
        self.h = lib().oc_create(ctypes.byref(cfg))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oc_destroy(self.h)
            self.h = None

    def init(self):
        lib().oc_init(self.h)

    def step(self, n: int = 1) -> int:
        return lib().oc_step(self.h, int(n))

    def regrid(self):
        lib().oc_regrid(self.h)

    def scalars(self) -> dict:
        out = np.zeros(17)
        lib().oc_scalars(self.h, _ptr(out))
        keys = ["t", "dt", "it", "ntrack", "nact", "iLbnd", "iRbnd", "cap", "tstart", "RShock",
                "Nalpha", "Nmp", "Nme", "rhoNorm", "pNorm", "lNorm", "lfacShock2"]
        return dict(zip(keys, out.tolist()))

    def snapshot(self) -> Snapshot:
        sc = self.scalars()
        cap = int(sc["cap"])
        prim = np.zeros((self.nq, cap))
        arrs = [np.zeros(cap) for _ in range(6)]
        xI = np.zeros(cap)
        n = lib().oc_snapshot(self.h, _ptr(prim), *[_ptr(a) for a in arrs], _ptr(xI), cap)
        return Snapshot(t=sc["t"], dt=sc["dt"], it=int(sc["it"]), ntrack=n,
                        prim=prim[:, :n].copy(), x=arrs[0][:n].copy(), dx=arrs[1][:n].copy(),
                        dt_loc=arrs[2][:n].copy(), sd=arrs[3][:n].copy(), pspec=arrs[4][:n].copy(),
                        shocked=arrs[5][:n].copy(), xI=xI[: n - 1].copy())

    def load(self, snap: Snapshot):
        n = snap.ntrack
        prim = np.ascontiguousarray(snap.prim[:, :n], dtype=np.float64)
        rc = lib().oc_load(self.h, n, _ptr(prim), _ptr(np.ascontiguousarray(snap.x)),
                           _ptr(np.ascontiguousarray(snap.dx)), _ptr(np.ascontiguousarray(snap.dt_loc)),
                           _ptr(np.ascontiguousarray(snap.xI)), n, float(snap.t), int(snap.it))
        if rc != 0:
            raise ValueError("track does not fit the oracle's capacity")

    def cons2prim(self, cons, prim_guess, r=None):
        cons = np.ascontiguousarray(cons, dtype=np.float64).copy()
        prim = np.ascontiguousarray(prim_guess, dtype=np.float64).copy()
        n = cons.shape[1]
        iters = (ctypes.c_int * n)()
        rr = None if r is None else np.ascontiguousarray(r, dtype=np.float64)
        lib().oc_cons2prim(self.h, _ptr(cons), _ptr(prim), _ptr(rr), n, iters)
        return prim, cons, np.frombuffer(iters, dtype=np.int32).copy()

    def prim2cons(self, prim, r=None):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        cons = np.zeros_like(prim)
        rr = None if r is None else np.ascontiguousarray(r, dtype=np.float64)
        lib().oc_prim2cons(self.h, _ptr(prim), _ptr(cons), _ptr(rr), prim.shape[1])
        return cons

    def riemann(self, primL, primR, x, v=None):
        primL = np.ascontiguousarray(primL, dtype=np.float64)
        primR = np.ascontiguousarray(primR, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = primL.shape[1]
        vv = np.zeros(n) if v is None else np.ascontiguousarray(v, dtype=np.float64)
        lam = np.zeros(3 * n)
        flux = np.zeros((self.nq, n))
        lib().oc_riemann(self.h, _ptr(primL), _ptr(primR), _ptr(x), _ptr(vv), 0 if v is None else 1,
                         _ptr(lam), _ptr(flux), n)
        return lam.reshape(n, 3), flux

    def bm_profile(self, r, t):
        r = np.ascontiguousarray(r, dtype=np.float64)
        rho, u, p = np.zeros_like(r), np.zeros_like(r), np.zeros_like(r)
        lib().oc_bm_profile(self.h, _ptr(r), r.size, float(t), _ptr(rho), _ptr(u), _ptr(p))
        return rho, u, p
