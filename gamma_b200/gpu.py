"""ctypes binding of the C ABI in include/gamma_gpu.h (gamma_b200/lib/libgamma_b200.so).

There is no CPU fallback: importing works everywhere, but creating a context
raises if the library is missing or no sm_100 device is present.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, fields

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GAMMA_B200_LIB") or os.path.join(HERE, "lib", "libgamma_b200.so")

GAMMA_OK = 0
GAMMA_ERR_INVALID = -1
GAMMA_ERR_CUDA = -2
GAMMA_ERR_CAPACITY = -3
GAMMA_ERR_NO_DEVICE = -4
GAMMA_ERR_NEG_DT = -30

GEOM_SPHERICAL1D, GEOM_CARTESIAN = 0, 1
HYDRO_REL_SPH, HYDRO_REL_CART, HYDRO_REL_CYL = 0, 1, 2
EOS_IDEAL, EOS_SYNGE = 0, 1
PROBLEM_BM1D, PROBLEM_TUBE = 0, 1
TS_RK3, TS_EULER = 0, 1  # Timestep/rk3.cpp, Timestep/euler.cpp

# every symbol include/gamma_gpu.h declares
EXPORTS = (
    "gamma_gpu_create", "gamma_gpu_layout", "gamma_gpu_set_params", "gamma_gpu_upload", "gamma_gpu_step",
    "gamma_gpu_regrid", "gamma_gpu_step_tubes_noalloc",
    "gamma_gpu_download", "gamma_gpu_cons2prim", "gamma_gpu_stream", "gamma_gpu_strerror",
    "gamma_gpu_last_error", "gamma_gpu_destroy",
    "gamma_mlp_param_count", "gamma_mlp_init", "gamma_mlp_pairs", "gamma_mlp_train", "gamma_mlp_forward",
    "gamma_mlp_loss_grad",
    "gamma_gpu_cons2prim_guess", "gamma_gpu_set_guess",
    "gamma_text1d_write", "gamma_text1d_read", "gamma_gpu_print_cols", "gamma_gpu_save", "gamma_gpu_load",
    "gamma_gpu_variant_info", "gamma_gpu_set_variant", "gamma_gpu_get_variant", "gamma_gpu_autotune",
    "gamma_gpu_use_graphs", "gamma_gpu_problem_id", "gamma_gpu_set_params_words", "gamma_gpu_initial_state",
)
PARAM_WORDS = 32  # gamma_problem::PARAM_WORDS


class GammaError(RuntimeError):
    def __init__(self, code: int, detail: str = ""):
        self.code = code
        super().__init__(f"{strerror(code)} ({code}){': ' + detail if detail else ''}")


class Config(ctypes.Structure):
    """gamma_config_t"""

    _fields_ = [(n, ctypes.c_int) for n in ("geometry", "hydro", "eos", "nq", "shock_detection",
                                             "local_synchrotron", "problem", "ngst")] + \
               [(n, ctypes.c_double) for n in ("gamma_ad", "cfl", "vi")] + \
               [("eos_wavespeeds", ctypes.c_int), ("timestep", ctypes.c_int)]


class RunParams(ctypes.Structure):
    """gamma_run_params_t"""

    _fields_ = [(n, ctypes.c_double) for n in (
        "Etot", "n_ext", "eta", "k", "Rscale", "rhoNorm", "pNorm", "lNorm", "vNorm", "dth", "target_ar",
        "split_AR", "merge_AR", "t_bm_until", "v_in", "v_out", "Nalpha", "Nmp", "Nme")]


class StepStats(ctypes.Structure):
    """gamma_step_stats_t"""

    _fields_ = [(n, ctypes.c_ulonglong) for n in ("c2p_calls", "c2p_iters", "c2p_fallbacks", "zone_updates",
                                                  "splits", "merges")] + \
               [("c2p_max_iters", ctypes.c_int), ("status", ctypes.c_int), ("device_ms", ctypes.c_float),
                ("c2p_guesses", ctypes.c_ulonglong), ("c2p_poor", ctypes.c_ulonglong),
                ("learned_steps", ctypes.c_ulonglong)]

    def as_dict(self) -> dict:
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class MlpTrain(ctypes.Structure):
    """gamma_mlp_train_t"""

    _fields_ = [("epochs", ctypes.c_int), ("batch", ctypes.c_int), ("lr", ctypes.c_float),
                ("lr_final", ctypes.c_float), ("seed", ctypes.c_ulonglong)]


def config_sph(gamma_ad=4. / 3., cfl=0.2, vi=1.0, eos=EOS_IDEAL, eos_wavespeeds=0, timestep=TS_RK3) -> Config:
    """spherical1D + rel_sph + radiation_sph, shock detection and local synchrotron (NUM_Q = 10).
    eos_wavespeeds=1 puts each state's Gamma_eff into the wave speeds and the
    shock detector too (the reference uses GAMMA_ there).  timestep: TS_RK3 or
    TS_EULER, the reference's Timestep module."""
    return Config(GEOM_SPHERICAL1D, HYDRO_REL_SPH, eos, 10, 1, 1, PROBLEM_BM1D, 2, gamma_ad, cfl, vi,
                  int(eos_wavespeeds), int(timestep))


def config_cart(gamma_ad=5. / 3., cfl=0.2, vi=1.0, timestep=TS_RK3, problem=PROBLEM_TUBE) -> Config:
    """cartesian + rel_cart, no shock detection or synchrotron (NUM_Q = 6).
    problem: a problem module's id (problem_id) running with these modules."""
    return Config(GEOM_CARTESIAN, HYDRO_REL_CART, EOS_IDEAL, 6, 0, 0, int(problem), 2, gamma_ad, cfl, vi, 0,
                  int(timestep))


def config_cyl(gamma_ad=5. / 3., cfl=0.2, vi=1.0, timestep=TS_RK3, problem=None) -> Config:
    """cartesian + rel_cyl (Hydro/rel_cyl.cpp), no shock detection or synchrotron
    (NUM_Q = 6); problem: a module built for it (default: tube_cyl)."""
    pid = problem_id("tube_cyl") if problem is None else int(problem)
    return Config(GEOM_CARTESIAN, HYDRO_REL_CYL, EOS_IDEAL, 6, 0, 0, pid, 2, gamma_ad, cfl, vi, 0, int(timestep))


def problem_id(name: str) -> int:
    """gamma_gpu_problem_id: the id of a problem module compiled into the library."""
    pid = lib().gamma_gpu_problem_id(name.encode())
    if pid < 0:
        raise KeyError(f"no problem module {name!r} in {LIB_PATH}")
    return pid


def initial_state(cfg: Config, words, cap: int):
    """gamma_gpu_initial_state: Simu::initialise of one run from the problem
    module's set-up hooks, on the host.  Returns (ntrack, t, prim [nq][cap], x,
    dx, xI, dt_loc)."""
    w = np.ascontiguousarray(words, dtype=np.float64)
    prim = np.zeros((cfg.nq, cap))
    x, dx, xI, dtl = np.zeros(cap), np.zeros(cap), np.zeros(cap), np.zeros(cap)
    nt, t = ctypes.c_int(), ctypes.c_double()
    rc = lib().gamma_gpu_initial_state(ctypes.byref(cfg), _p(w), int(w.size), int(cap), ctypes.byref(nt),
                                       ctypes.byref(t), _p(prim), _p(x), _p(dx), _p(xI), _p(dtl))
    if rc != GAMMA_OK:
        raise GammaError(rc)
    return int(nt.value), float(t.value), prim, x, dx, xI, dtl


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_longlong)
_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                                    f"(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.gamma_gpu_create.argtypes = [ctypes.POINTER(Config), ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_void_p)]
        L.gamma_gpu_layout.argtypes = [ctypes.c_void_p, _lp, _lp]
        L.gamma_gpu_set_params.argtypes = [ctypes.c_void_p, ctypes.POINTER(RunParams)]
        L.gamma_gpu_upload.argtypes = [ctypes.c_void_p, _ip, _dp, _lp, _dp, _dp, _dp, _dp, _dp]
        L.gamma_gpu_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(StepStats)]
        L.gamma_gpu_regrid.argtypes = [ctypes.c_void_p, ctypes.POINTER(StepStats)]
        L.gamma_gpu_download.argtypes = [ctypes.c_void_p, _ip, _dp, _dp, _lp, _ip, _dp, _dp, _dp, _dp, _dp]
        L.gamma_gpu_cons2prim.argtypes = [ctypes.POINTER(Config), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p]
        L.gamma_gpu_step_tubes_noalloc.argtypes = [ctypes.POINTER(Config), ctypes.c_int, ctypes.c_longlong] + \
            [ctypes.c_void_p] * 8 + [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(StepStats)]
        L.gamma_gpu_step_tubes_noalloc.restype = ctypes.c_int
        L.gamma_gpu_stream.restype = ctypes.c_void_p
        L.gamma_gpu_stream.argtypes = [ctypes.c_void_p]
        L.gamma_gpu_strerror.restype = ctypes.c_char_p
        L.gamma_gpu_strerror.argtypes = [ctypes.c_int]
        L.gamma_gpu_last_error.restype = ctypes.c_char_p
        L.gamma_gpu_last_error.argtypes = [ctypes.c_void_p]
        L.gamma_gpu_destroy.argtypes = [ctypes.c_void_p]
        v = ctypes.c_void_p
        L.gamma_mlp_param_count.argtypes = []
        L.gamma_mlp_init.argtypes = [v, ctypes.c_ulonglong, v]
        L.gamma_mlp_pairs.argtypes = [ctypes.POINTER(Config), v, ctypes.c_longlong, ctypes.c_longlong,
                                      ctypes.c_ulonglong, v, v, v]
        L.gamma_mlp_train.argtypes = [v, v, v, ctypes.c_longlong, ctypes.POINTER(MlpTrain),
                                      ctypes.POINTER(ctypes.c_float), v]
        L.gamma_mlp_forward.argtypes = [v, v, ctypes.c_longlong, v, ctypes.c_int, v]
        L.gamma_mlp_loss_grad.argtypes = [v, v, v, ctypes.c_int, v, v, v]
        L.gamma_gpu_cons2prim_guess.argtypes = [ctypes.POINTER(Config), v, v, ctypes.c_int, v, v, v]
        L.gamma_gpu_set_guess.argtypes = [v, v]
        L.gamma_text1d_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config), ctypes.c_int, ctypes.c_longlong,
                                         ctypes.c_double, _dp, ctypes.c_longlong, _dp, _dp]
        L.gamma_text1d_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config), ctypes.c_int, _ip, _lp, _dp,
                                        _dp, _dp, _dp, _dp]
        L.gamma_gpu_print_cols.argtypes = [v, ctypes.c_int, ctypes.c_char_p]
        L.gamma_gpu_variant_info.argtypes = [ctypes.c_int, _ip, _ip]
        L.gamma_gpu_set_variant.argtypes = [v, ctypes.c_int]
        L.gamma_gpu_get_variant.argtypes = [v]
        L.gamma_gpu_autotune.argtypes = [v, ctypes.c_int, ctypes.POINTER(ctypes.c_float), _ip]
        L.gamma_gpu_use_graphs.argtypes = [v, ctypes.c_int]
        L.gamma_gpu_save.argtypes = [v, ctypes.c_char_p]
        L.gamma_gpu_problem_id.argtypes = [ctypes.c_char_p]
        L.gamma_gpu_set_params_words.argtypes = [v, _dp, ctypes.c_int]
        L.gamma_gpu_initial_state.argtypes = [ctypes.POINTER(Config), _dp, ctypes.c_int, ctypes.c_int, _ip, _dp,
                                              _dp, _dp, _dp, _dp, _dp]
        L.gamma_gpu_load.argtypes = [v, ctypes.c_char_p]
        for name in ("gamma_gpu_create", "gamma_gpu_layout", "gamma_gpu_set_params", "gamma_gpu_upload",
                     "gamma_gpu_step", "gamma_gpu_regrid", "gamma_gpu_download", "gamma_gpu_cons2prim",
                     "gamma_mlp_param_count", "gamma_mlp_init", "gamma_mlp_pairs", "gamma_mlp_train",
                     "gamma_mlp_forward", "gamma_gpu_cons2prim_guess", "gamma_gpu_set_guess", "gamma_mlp_loss_grad",
                     "gamma_text1d_write", "gamma_text1d_read", "gamma_gpu_print_cols", "gamma_gpu_save",
                     "gamma_gpu_load", "gamma_gpu_variant_info", "gamma_gpu_set_variant", "gamma_gpu_get_variant",
                     "gamma_gpu_autotune", "gamma_gpu_use_graphs", "gamma_gpu_problem_id",
                     "gamma_gpu_set_params_words", "gamma_gpu_initial_state"):
            getattr(L, name).restype = ctypes.c_int
        _LIB = L
    return _LIB


def strerror(code: int) -> str:
    return lib().gamma_gpu_strerror(int(code)).decode()


def _p(a, typ=_dp):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(typ)


class GammaGPU:
    """One context: nruns independent tracks on the current CUDA device."""

    def __init__(self, cfg: Config, capacities):
        self.cfg = cfg
        self.nq = cfg.nq
        caps = np.ascontiguousarray(capacities, dtype=np.int32)
        self.nruns = caps.size
        self.cap = caps
        h = ctypes.c_void_p()
        rc = lib().gamma_gpu_create(ctypes.byref(cfg), self.nruns, _p(caps, _ip), ctypes.byref(h))
        if rc != GAMMA_OK:
            raise GammaError(rc)
        self.h = h
        self._destroy = lib().gamma_gpu_destroy  # bound now: module globals may be gone when __del__ runs
        offs = np.zeros(self.nruns, dtype=np.int64)
        tot = ctypes.c_longlong()
        lib().gamma_gpu_layout(self.h, _p(offs, _lp), ctypes.byref(tot))
        self.offsets = offs
        self.total = int(tot.value)

    def _check(self, rc):
        if rc != GAMMA_OK:
            raise GammaError(rc, lib().gamma_gpu_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def stream(self) -> int:
        return lib().gamma_gpu_stream(self.h)

    def set_params(self, params):
        arr = (RunParams * self.nruns)(*params)
        self._check(lib().gamma_gpu_set_params(self.h, arr))

    def set_params_words(self, words):
        """The problem module's parameter words of every run ([nruns][nwords], nwords <= PARAM_WORDS)."""
        w = np.ascontiguousarray(np.atleast_2d(words), dtype=np.float64)
        assert w.shape[0] == self.nruns
        self._check(lib().gamma_gpu_set_params_words(self.h, _p(w), int(w.shape[1])))

    def upload(self, ntrack, prim, x, dx, xI, dt_loc=None, t=None, it=None):
        nt = np.ascontiguousarray(ntrack, dtype=np.int32)
        tt = None if t is None else np.ascontiguousarray(t, dtype=np.float64)
        ii = None if it is None else np.ascontiguousarray(it, dtype=np.int64)
        self._check(lib().gamma_gpu_upload(self.h, _p(nt, _ip), _p(tt), _p(ii, _lp), _p(prim), _p(x), _p(dx),
                                           _p(dt_loc), _p(xI)))

    def upload_ptrs(self, ntrack, t, it, prim_ptr, x_ptr, dx_ptr, dtl_ptr, xI_ptr):
        """Upload from raw host addresses (e.g. pinned torch tensors)."""
        nt = np.ascontiguousarray(ntrack, dtype=np.int32)
        tt = np.ascontiguousarray(t, dtype=np.float64)
        ii = np.ascontiguousarray(it, dtype=np.int64)
        c = lambda v: ctypes.cast(ctypes.c_void_p(v), _dp) if v else None
        self._check(lib().gamma_gpu_upload(self.h, _p(nt, _ip), _p(tt), _p(ii, _lp), c(prim_ptr), c(x_ptr),
                                           c(dx_ptr), c(dtl_ptr), c(xI_ptr)))

    def step(self, nsteps: int = 1, stats: bool = True):
        st = StepStats()
        self._check(lib().gamma_gpu_step(self.h, int(nsteps), ctypes.byref(st) if stats else None))
        return st.as_dict() if stats else None

    def set_guess(self, params_ptr: int):
        """Learned cons2prim starting pressure in every step (device parameter
        pointer), or 0 for the warm start of the reference."""
        self._check(lib().gamma_gpu_set_guess(self.h, ctypes.c_void_p(params_ptr) if params_ptr else None))

    def regrid(self):
        st = StepStats()
        self._check(lib().gamma_gpu_regrid(self.h, ctypes.byref(st)))
        return st.as_dict()

    def download(self) -> dict:
        R, N = self.nruns, self.total
        out = dict(ntrack=np.zeros(R, np.int32), t=np.zeros(R), dt=np.zeros(R), it=np.zeros(R, np.int64),
                   status=np.zeros(R, np.int32), prim=np.zeros((self.nq, N)), x=np.zeros(N), dx=np.zeros(N),
                   dt_loc=np.zeros(N), xI=np.zeros(N))
        self._check(lib().gamma_gpu_download(
            self.h, _p(out["ntrack"], _ip), _p(out["t"]), _p(out["dt"]), _p(out["it"], _lp), _p(out["status"], _ip),
            _p(out["prim"]), _p(out["x"]), _p(out["dx"]), _p(out["dt_loc"]), _p(out["xI"])))
        return out

    def print_cols(self, run: int, directory: str) -> str:
        """Grid::printCols of one run: marks isShocked into slot TR1+1 on the
        device (as the reference does), writes <directory>/phys%010d.out and
        returns that path."""
        self._check(lib().gamma_gpu_print_cols(self.h, int(run), directory.encode()))
        it = int(self.download()["it"][run])
        return os.path.join(directory, f"phys{it:010d}.out")

    def use_graphs(self, on: bool):
        """Replay step calls from a captured CUDA graph (default) or launch directly."""
        self._check(lib().gamma_gpu_use_graphs(self.h, 1 if on else 0))

    def set_variant(self, variant: int):
        """Launch shape of the step kernel (variant_info); results do not change."""
        self._check(lib().gamma_gpu_set_variant(self.h, int(variant)))

    @property
    def variant(self) -> int:
        return int(lib().gamma_gpu_get_variant(self.h))

    def autotune(self, nsteps: int = 3):
        """Times nsteps steps of every launch shape on the current state (which
        it restores) and keeps the fastest; returns (ms per variant, chosen)."""
        ms = (ctypes.c_float * N_VARIANTS)()
        ch = ctypes.c_int()
        self._check(lib().gamma_gpu_autotune(self.h, int(nsteps), ms, ctypes.byref(ch)))
        return [float(x) for x in ms], int(ch.value)

    def save(self, path: str):
        """Exact checkpoint of every run."""
        self._check(lib().gamma_gpu_save(self.h, path.encode()))

    def load(self, path: str):
        """Restore a checkpoint made by a context of the same configuration and capacities."""
        self._check(lib().gamma_gpu_load(self.h, path.encode()))

    def download_ptrs(self, prim_ptr, x_ptr=None, dx_ptr=None, dtl_ptr=None, xI_ptr=None):
        R = self.nruns
        nt = np.zeros(R, np.int32)
        c = lambda v: ctypes.cast(ctypes.c_void_p(v), _dp) if v else None
        self._check(lib().gamma_gpu_download(self.h, _p(nt, _ip), None, None, None, None, c(prim_ptr), c(x_ptr),
                                             c(dx_ptr), c(dtl_ptr), c(xI_ptr)))
        return nt


N_VARIANTS = 8


def variant_info(variant: int):
    """(threads per run, cells per thread per sweep chunk) of a launch shape."""
    a, b = ctypes.c_int(), ctypes.c_int()
    _ok(lib().gamma_gpu_variant_info(int(variant), ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def text1d_write(path: str, cfg: Config, prim, x, dx, it: int, t: float):
    """Grid::printCols columns of one run from host arrays: prim [nq][ntrack]
    (slot TR1+1 already holding what the reference stores there), x, dx."""
    prim = np.ascontiguousarray(prim, dtype=np.float64)
    n = prim.shape[1]
    _ok(lib().gamma_text1d_write(path.encode(), ctypes.byref(cfg), int(n), int(it), float(t), _p(prim), int(n),
                                 _p(np.ascontiguousarray(x, dtype=np.float64)),
                                 _p(np.ascontiguousarray(dx, dtype=np.float64))))


def text1d_read(path: str, cfg: Config, cap: int) -> dict:
    """Simu::reinitialise of the 1D build without the problem hooks: the state
    reloadFromData + mpi_distribute + prepForRun leave ([nq][cap] arrays;
    ghost cells still to be filled by the problem's updateGhosts)."""
    prim = np.zeros((cfg.nq, cap))
    x, dx, xI = np.zeros(cap), np.zeros(cap), np.zeros(cap)
    n = ctypes.c_int()
    it = ctypes.c_longlong()
    t = ctypes.c_double()
    _ok(lib().gamma_text1d_read(path.encode(), ctypes.byref(cfg), int(cap), ctypes.byref(n), ctypes.byref(it),
                                ctypes.byref(t), _p(prim), _p(x), _p(dx), _p(xI)))
    return dict(ntrack=int(n.value), it=int(it.value), t=float(t.value), prim=prim, x=x, dx=dx, xI=xI)


def cons2prim_device(cfg: Config, cons_ptr: int, prim_ptr: int, n: int, iters_ptr: int = 0, stream: int = 0):
    """FluidState::cons2prim on device arrays [nq][n] (raw CUDA pointers)."""
    rc = lib().gamma_gpu_cons2prim(ctypes.byref(cfg), ctypes.c_void_p(cons_ptr), ctypes.c_void_p(prim_ptr), int(n),
                                   ctypes.c_void_p(iters_ptr) if iters_ptr else None,
                                   ctypes.c_void_p(stream) if stream else None)
    if rc != GAMMA_OK:
        raise GammaError(rc)


class RunState(ctypes.Structure):
    """gamma_run_state_t"""

    _fields_ = [("ntrack", ctypes.c_int), ("status", ctypes.c_int), ("t", ctypes.c_double),
                ("dt", ctypes.c_double), ("it", ctypes.c_longlong)]


def step_tubes_noalloc(cfg: Config, nruns: int, total: int, offsets_ptr: int, capacity_ptr: int, runs_ptr: int,
                       prim_ptr: int, x_ptr: int, dx_ptr: int, dtl_ptr: int, xI_ptr: int, nsteps: int,
                       stream: int = 0, stats: bool = True):
    """gamma_gpu_step_tubes_noalloc on caller-owned device arrays (raw CUDA pointers)."""
    st = StepStats()
    v = ctypes.c_void_p
    rc = lib().gamma_gpu_step_tubes_noalloc(ctypes.byref(cfg), int(nruns), int(total), v(offsets_ptr),
                                            v(capacity_ptr), v(runs_ptr), v(prim_ptr), v(x_ptr), v(dx_ptr),
                                            v(dtl_ptr), v(xI_ptr), int(nsteps), v(stream) if stream else None,
                                            ctypes.byref(st) if stats else None)
    if rc != GAMMA_OK:
        raise GammaError(rc)
    return st.as_dict() if stats else None


def _ok(rc):
    if rc != GAMMA_OK:
        raise GammaError(rc)


def mlp_param_count() -> int:
    return int(lib().gamma_mlp_param_count())


def mlp_init(params_ptr: int, seed: int, stream: int = 0):
    _ok(lib().gamma_mlp_init(ctypes.c_void_p(params_ptr), ctypes.c_ulonglong(seed),
                             ctypes.c_void_p(stream) if stream else None))


def mlp_pairs(cfg: Config, prim_ptr: int, n_states: int, n_uniform: int, seed: int, x_ptr: int, y_ptr: int,
              stream: int = 0):
    """Training pairs (x [n][3], y [n][2] floats) from n_states device primitive
    states [nq][n_states] followed by n_uniform drawn states."""
    _ok(lib().gamma_mlp_pairs(ctypes.byref(cfg), ctypes.c_void_p(prim_ptr) if prim_ptr else None, int(n_states),
                              int(n_uniform), ctypes.c_ulonglong(seed), ctypes.c_void_p(x_ptr),
                              ctypes.c_void_p(y_ptr), ctypes.c_void_p(stream) if stream else None))


def mlp_train(params_ptr: int, x_ptr: int, y_ptr: int, n: int, epochs: int = 8, batch: int = 8192,
              lr: float = 3e-3, lr_final: float = 1e-4, seed: int = 7, stream: int = 0) -> np.ndarray:
    """Mini-batch Adam; returns the mean training loss of each epoch."""
    tc = MlpTrain(int(epochs), int(batch), float(lr), float(lr_final), int(seed))
    loss = np.zeros(max(int(epochs), 1), dtype=np.float32)
    _ok(lib().gamma_mlp_train(ctypes.c_void_p(params_ptr), ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), int(n),
                              ctypes.byref(tc), loss.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                              ctypes.c_void_p(stream) if stream else None))
    return loss[:int(epochs)]


def mlp_loss_grad(params_ptr: int, x_ptr: int, y_ptr: int, n: int, grad_ptr: int, loss_ptr: int = 0,
                  stream: int = 0):
    """Gradient (and loss) of the training objective over n samples, on device arrays."""
    _ok(lib().gamma_mlp_loss_grad(ctypes.c_void_p(params_ptr), ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                  int(n), ctypes.c_void_p(grad_ptr), ctypes.c_void_p(loss_ptr) if loss_ptr else None,
                                  ctypes.c_void_p(stream) if stream else None))


def mlp_forward(params_ptr: int, x_ptr: int, n: int, out_ptr: int, tensor_cores: bool, stream: int = 0):
    _ok(lib().gamma_mlp_forward(ctypes.c_void_p(params_ptr), ctypes.c_void_p(x_ptr), int(n), ctypes.c_void_p(out_ptr),
                                1 if tensor_cores else 0, ctypes.c_void_p(stream) if stream else None))


def cons2prim_guess_device(cfg: Config, cons_ptr: int, prim_ptr: int, n: int, params_ptr: int, iters_ptr: int = 0,
                           stream: int = 0):
    """cons2prim on device arrays [nq][n] started from the network's pressure."""
    _ok(lib().gamma_gpu_cons2prim_guess(ctypes.byref(cfg), ctypes.c_void_p(cons_ptr), ctypes.c_void_p(prim_ptr),
                                        int(n), ctypes.c_void_p(iters_ptr) if iters_ptr else None,
                                        ctypes.c_void_p(params_ptr), ctypes.c_void_p(stream) if stream else None))
