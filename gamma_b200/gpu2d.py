"""ctypes binding of the 2D (r, theta) step (gamma_2d_* in include/gamma_gpu.h).

The state of a run is a :class:`State2D` of flat numpy arrays in the C ABI's
layout: NJ = ntheta + 2 ngst tracks (ghost tracks included) of ``cap`` cells,
cell (j, i) at j * cap + i.  There is no CPU fallback: every call goes to the
CUDA library.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import gpu

NQ = 10


class Config2D(ctypes.Structure):
    """gamma_2d_config_t"""

    _fields_ = [("ntheta", ctypes.c_int), ("nmax", ctypes.c_int), ("ngst", ctypes.c_int), ("nq", ctypes.c_int),
                ("eos", ctypes.c_int), ("gamma_ad", ctypes.c_double), ("cfl", ctypes.c_double),
                ("vi", ctypes.c_double), ("eos_wavespeeds", ctypes.c_int), ("timestep", ctypes.c_int)]


class Params2D(ctypes.Structure):
    """gamma_2d_params_t"""

    _fields_ = [(n, ctypes.c_double) for n in ("split_DR", "merge_DR", "split_DR_slow", "merge_DR_slow", "v_out",
                                                 "it_hold", "Nalpha", "Nmp", "Nme")]


@dataclass
class State2D:
    """A 2D run in the ABI layout (arrays over NJ * cap cells)."""

    NJ: int
    cap: int
    ntrack: np.ndarray            # [NJ] int32
    prim: np.ndarray              # [NQ, NJ*cap]
    x: np.ndarray                 # r
    dx: np.ndarray                # dr
    xI: np.ndarray                # interface r (right edge of each cell)
    dt_loc: np.ndarray | None = None
    grad_mv: np.ndarray | None = None
    grad_f1: np.ndarray | None = None
    nbr: np.ndarray | None = None  # [4, NJ*cap] int32
    t: float = 0.
    it: int = 0
    extra: dict = field(default_factory=dict)

    def track(self, j: int) -> dict:
        o, n = j * self.cap, int(self.ntrack[j])
        out = dict(n=n, prim=self.prim[:, o:o + n], x=self.x[o:o + n], dx=self.dx[o:o + n],
                   xI=self.xI[o:o + n - 1])
        for k in ("dt_loc",):
            v = getattr(self, k)
            if v is not None:
                out[k] = v[o:o + n]
        for k, v in self.extra.items():
            out[k] = v[..., o:o + n]
        return out


_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        L = gpu.lib()
        v = ctypes.c_void_p
        L.gamma_2d_create.argtypes = [ctypes.POINTER(Config2D), v, v, ctypes.POINTER(ctypes.c_void_p)]
        L.gamma_2d_layout.argtypes = [v, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.gamma_2d_set_params.argtypes = [v, ctypes.POINTER(Params2D)]
        L.gamma_2d_set_guess.argtypes = [v, v]
        L.gamma_2d_print_cols.argtypes = [v, ctypes.c_char_p]
        L.gamma_2d_save.argtypes = [v, ctypes.c_char_p]
        L.gamma_2d_load.argtypes = [v, ctypes.c_char_p]
        L.gamma_text2d_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config2D), v, v, v, ctypes.c_longlong,
                                         ctypes.c_double, v, v, v]
        L.gamma_text2d_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config2D), v, v, v, v, v, v, v, v, v]
        L.gamma_2d_upload.argtypes = [v] + [v] * 9 + [ctypes.c_double, ctypes.c_longlong, ctypes.c_int]
        L.gamma_2d_step.argtypes = [v, ctypes.c_int, ctypes.POINTER(gpu.StepStats)]
        L.gamma_2d_use_graphs.argtypes = [v, ctypes.c_int]
        L.gamma_2d_use_graphs.restype = ctypes.c_int
        L.gamma_2d_download.argtypes = [v] * 17
        L.gamma_2d_prepare.argtypes = [v]
        L.gamma_2d_prepare_stage.argtypes = [v, ctypes.c_int]
        L.gamma_2d_prepare_stage.restype = ctypes.c_int
        L.gamma_2d_download_fluxes.argtypes = [v] * 8
        L.gamma_2d_stream.argtypes = [v]
        L.gamma_2d_stream.restype = v
        L.gamma_2d_last_error.argtypes = [v]
        L.gamma_2d_last_error.restype = ctypes.c_char_p
        L.gamma_2d_destroy.argtypes = [v]
        for name in ("gamma_2d_create", "gamma_2d_layout", "gamma_2d_set_params", "gamma_2d_set_guess",
                     "gamma_2d_upload", "gamma_2d_step", "gamma_2d_download", "gamma_2d_prepare",
                     "gamma_2d_download_fluxes", "gamma_2d_print_cols", "gamma_2d_save", "gamma_2d_load",
                     "gamma_text2d_write", "gamma_text2d_read"):
            getattr(L, name).restype = ctypes.c_int
        _LIB = L
    return _LIB


def _ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


class Grid2DGPU:
    """One 2D run on the current CUDA device."""

    def __init__(self, ntheta: int, nmax: int, theta, dtheta, gamma_ad=4. / 3., cfl=0.2, vi=1.0,
                 eos=gpu.EOS_IDEAL, eos_wavespeeds=0, timestep=gpu.TS_RK3):
        self.cfg = Config2D(int(ntheta), int(nmax), 2, NQ, int(eos), float(gamma_ad), float(cfl), float(vi),
                            int(eos_wavespeeds), int(timestep))
        th = np.ascontiguousarray(theta, dtype=np.float64)
        dth = np.ascontiguousarray(dtheta, dtype=np.float64)
        assert th.size == ntheta and dth.size == ntheta
        h = ctypes.c_void_p()
        rc = lib().gamma_2d_create(ctypes.byref(self.cfg), _ptr(th), _ptr(dth), ctypes.byref(h))
        if rc != gpu.GAMMA_OK:
            raise gpu.GammaError(rc)
        self.h = h
        self._destroy = lib().gamma_2d_destroy  # bound now: module globals may be gone when __del__ runs
        nj, cap = ctypes.c_int(), ctypes.c_int()
        lib().gamma_2d_layout(self.h, ctypes.byref(nj), ctypes.byref(cap))
        self.NJ, self.cap = nj.value, cap.value
        self.NC = self.NJ * self.cap

    def _check(self, rc):
        if rc != gpu.GAMMA_OK:
            raise gpu.GammaError(rc, lib().gamma_2d_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def stream(self) -> int:
        return lib().gamma_2d_stream(self.h)

    def set_params(self, p: Params2D):
        self._check(lib().gamma_2d_set_params(self.h, ctypes.byref(p)))

    def use_graphs(self, on: bool):
        """Each step replayed from a captured CUDA graph (default), or its
        kernels launched one by one."""
        self._check(lib().gamma_2d_use_graphs(self.h, int(bool(on))))

    def set_guess(self, params_ptr: int):
        """Learned cons2prim starting pressure in every cell update (device
        parameter pointer), or 0 for the warm start of the reference."""
        self._check(lib().gamma_2d_set_guess(self.h, ctypes.c_void_p(params_ptr) if params_ptr else None))

    def upload(self, s: State2D, run_ghosts: bool = False):
        assert s.NJ == self.NJ and s.cap == self.cap
        c = lambda a, dt: None if a is None else np.ascontiguousarray(a, dtype=dt)
        arrs = [c(s.ntrack, np.int32), c(s.prim, np.float64), c(s.x, np.float64), c(s.dx, np.float64),
                c(s.dt_loc, np.float64), c(s.xI, np.float64), c(s.grad_mv, np.float64), c(s.grad_f1, np.float64),
                c(s.nbr, np.int32)]
        self._keep = arrs
        self._check(lib().gamma_2d_upload(self.h, *[_ptr(a) for a in arrs], float(s.t), int(s.it),
                                          1 if run_ghosts else 0))

    def step(self, nsteps: int = 1, stats: bool = True):
        st = gpu.StepStats()
        self._check(lib().gamma_2d_step(self.h, int(nsteps), ctypes.byref(st) if stats else None))
        return st.as_dict() if stats else None

    def prepare(self):
        """regrid, ghosts and the stage-1 fluxes only (diagnostics)"""
        self._check(lib().gamma_2d_prepare(self.h))

    def prepare_stage(self, stage: int):
        """gamma_2d_prepare_stage: the loop body up to stage `stage`'s fluxes."""
        self._check(lib().gamma_2d_prepare_stage(self.h, int(stage)))

    def download_fluxes(self) -> dict:
        NC = self.NC
        out = dict(v=np.zeros(NC), lL=np.zeros(NC), lR=np.zeros(NC), flux=np.zeros((NQ, NC)),
                   f1lo=np.zeros((NQ, NC)), f1hi=np.zeros((NQ, NC)), grad_f1=np.zeros((NQ, NC)))
        self._check(lib().gamma_2d_download_fluxes(self.h, *[_ptr(out[k]) for k in
                                                             ("v", "lL", "lR", "flux", "f1lo", "f1hi", "grad_f1")]))
        return out

    def print_cols(self, directory: str) -> str:
        """Grid::printCols of the 2D build: Sd into slot TR1+1 of every cell
        on the device (as the reference does), then <directory>/phys%010d.out;
        returns that path."""
        self._check(lib().gamma_2d_print_cols(self.h, directory.encode()))
        it = ctypes.c_longlong()
        self._check(lib().gamma_2d_download(self.h, *([None] * 3), ctypes.byref(it), *([None] * 12)))
        return f"{directory.rstrip('/')}/phys{it.value:010d}.out"

    def save(self, path: str):
        """Exact checkpoint (state, gradients, neighbour lists, dt_loc, t, it)."""
        self._check(lib().gamma_2d_save(self.h, path.encode()))

    def load(self, path: str):
        """Restore a checkpoint made with the same configuration and tracks."""
        self._check(lib().gamma_2d_load(self.h, path.encode()))

    def download(self) -> State2D:
        NC = self.NC
        nt = np.zeros(self.NJ, np.int32)
        t, dt, it, status = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong(), ctypes.c_int()
        prim = np.zeros((NQ, NC))
        x, dx, dtl, xI = (np.zeros(NC) for _ in range(4))
        gmv, gf1 = np.zeros((NQ, NC)), np.zeros((NQ, NC))
        nbr = np.zeros((4, NC), np.int32)
        sd, ps = np.zeros(NC), np.zeros(NC)
        sh = np.zeros(NC, np.uint8)
        self._check(lib().gamma_2d_download(
            self.h, _ptr(nt), ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it), ctypes.byref(status), _ptr(prim),
            _ptr(x), _ptr(dx), _ptr(dtl), _ptr(xI), _ptr(gmv), _ptr(gf1), _ptr(nbr), _ptr(sd), _ptr(ps), _ptr(sh)))
        s = State2D(self.NJ, self.cap, nt, prim, x, dx, xI, dtl, gmv, gf1, nbr, t.value, it.value,
                    extra=dict(sd=sd, pspec=ps, shocked=sh))
        s.extra["dt"] = np.array([dt.value])
        s.extra["status"] = np.array([status.value])
        return s


def _config(ntheta, nmax, gamma_ad=4. / 3., cfl=0.2, vi=1.0, eos=gpu.EOS_IDEAL, eos_wavespeeds=0,
            timestep=gpu.TS_RK3) -> Config2D:
    return Config2D(int(ntheta), int(nmax), 2, NQ, int(eos), float(gamma_ad), float(cfl), float(vi),
                    int(eos_wavespeeds), int(timestep))


def text2d_write(path: str, s: State2D, theta, dtheta, **cfg):
    """Grid::printCols columns of the 2D build from a host state whose slot
    TR1+1 already holds Sd; theta/dtheta of the active tracks."""
    c = _config(s.NJ - 4, s.cap - 4, **cfg)
    arr = lambda a, dt: np.ascontiguousarray(a, dtype=dt)
    keep = [arr(s.ntrack, np.int32), arr(theta, np.float64), arr(dtheta, np.float64), arr(s.prim, np.float64),
            arr(s.x, np.float64), arr(s.dx, np.float64)]
    gpu._ok(lib().gamma_text2d_write(path.encode(), ctypes.byref(c), _ptr(keep[0]), _ptr(keep[1]), _ptr(keep[2]),
                                     int(s.it), float(s.t), _ptr(keep[3]), _ptr(keep[4]), _ptr(keep[5])))


def text2d_read(path: str, ntheta: int, nmax: int, **cfg):
    """Simu::reinitialise of the 2D build: the state prepForRun leaves (ghost
    tracks and cells for the ghost pass), and the tracks' theta/dtheta."""
    c = _config(ntheta, nmax, **cfg)
    NJ, cap = ntheta + 4, nmax + 4
    NC = NJ * cap
    nt = np.zeros(NJ, np.int32)
    th, dth = np.zeros(ntheta), np.zeros(ntheta)
    prim = np.zeros((NQ, NC))
    x, dx, xI = np.zeros(NC), np.zeros(NC), np.zeros(NC)
    it, t = ctypes.c_longlong(), ctypes.c_double()
    gpu._ok(lib().gamma_text2d_read(path.encode(), ctypes.byref(c), _ptr(nt), ctypes.byref(it), ctypes.byref(t),
                                    _ptr(th), _ptr(dth), _ptr(prim), _ptr(x), _ptr(dx), _ptr(xI)))
    return State2D(NJ, cap, nt, prim, x, dx, xI, t=t.value, it=it.value), th, dth


EXPORTS = ("gamma_2d_create", "gamma_2d_layout", "gamma_2d_set_params", "gamma_2d_set_guess", "gamma_2d_upload",
           "gamma_2d_step",
           "gamma_2d_download", "gamma_2d_prepare", "gamma_2d_download_fluxes", "gamma_2d_stream",
           "gamma_2d_last_error", "gamma_2d_destroy", "gamma_2d_print_cols", "gamma_2d_save", "gamma_2d_load",
           "gamma_text2d_write", "gamma_text2d_read", "gamma_2d_use_graphs", "gamma_2d_prepare_stage")
