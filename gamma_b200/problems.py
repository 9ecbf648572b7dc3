"""Problem set-up on the host: the INITIAL modules of the reference.

The reference builds its initial track with the user hooks loadParams,
Grid::initialGeometry and Grid::initialValues, then Grid::prepForRun
(v2u, prim2cons, interfaceGeomFromCellPos, src/grid.cpp:20-26), the synchrotron
tracer initialisation (radiation_initGammas, radiation_sph.cpp:246-260) and one
updateGhosts (src/simu.cpp:74).  This module does the same for the two problem
families of this path and packs any number of runs into the pooled layout of
the C ABI (include/gamma_gpu.h).  Scalar maths uses Python's ``math`` (the C
library), so the states equal the reference's bit for bit.

Set-up runs once per job on the host; the step itself runs on the GPU.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import gpu

# src/constants.h
MP = 1.6726219e-24
ME = 9.1093835e-28
C_LIGHT = 2.99792458e10
ALPHA_SYN = 1.29251816e-09
PI = math.pi
DT_INF = 1.e15
RHO, PPP, UU1, UU2, TR1, GMN, GMX, GMD, PSN = 0, 1, 2, 3, 4, 6, 7, 8, 9


def _lfac(u):
    uu = 0.0
    uu += u * u
    uu = math.sqrt(uu)
    return math.sqrt(1 + uu * uu)


@dataclass
class TrackState:
    """One run: cells [0, ntrack), interfaces [0, ntrack-1)."""

    ntrack: int
    cap: int
    prim: np.ndarray   # [nq, ntrack]
    x: np.ndarray
    dx: np.ndarray
    xI: np.ndarray     # [ntrack-1]
    dt_loc: np.ndarray
    t: float = 0.0
    it: int = 0


def _default_prim(nq, n):
    p = np.zeros((nq, n))
    p[RHO] = 1.0
    p[PPP] = 1.0
    return p


def _prep_for_run(prim, x, dx, ngst):
    """v2u and interfaceGeomFromCellPos (src/Dimensions/1d.cpp:844-951)."""
    n = x.size
    u = prim[UU1]
    v = np.sqrt(0.0 + u * u)
    lfac = 1.0 / np.sqrt(1.0 - v * v)
    prim[UU1] = u * lfac
    iL = ngst - 1
    xI = x[:-1] + dx[:-1] / 2.0
    xI[iL] = x[iL + 1] - dx[iL + 1] / 2.0
    return xI


def _update_ghosts(prim, x, dx, xI, ngst):
    """Grid::updateGhosts without the user boundary hook (1d.cpp:217-246)."""
    n = x.size
    iL, iR = ngst - 1, n - ngst
    for i in range(0, iL + 1):
        prim[:, i] = prim[:, iL + 1]
        x[i] = x[iL + 1] - (iL - i + 1) * dx[iL + 1]
        dx[i] = dx[iL + 1]
    for i in range(0, iL):
        xI[i] = xI[iL + 1] - (iL - i + 1) * dx[iL + 1]
    for i in range(iR, n):
        prim[:, i] = prim[:, iR - 1]
        x[i] = x[iR - 1] + (i - iR + 1) * dx[iR - 1]
        dx[i] = dx[iR - 1]
    for i in range(iR, n - 1):
        xI[i] = xI[iR - 1] + (i - iR) * dx[iR - 1]


@dataclass
class TubeSetup:
    """Planar relativistic shock tube (cartesian + rel_cart), after src/Initial/Tests/1DST.cpp."""

    ncell: int = 1000
    nmax: int = 0          # 0: ncell (no regrid)
    ngst: int = 2
    xmin: float = 0.0
    xmax: float = 1.0
    xmid: float = 0.5
    rhoL: float = 10.0
    pL: float = 13.33
    vL: float = 0.0
    trL: float = 1.0
    rhoR: float = 1.0
    pR: float = 1.e-7
    vR: float = 0.0
    trR: float = 2.0

    nq = 6

    @property
    def capacity(self) -> int:
        return (self.nmax or self.ncell) + 2 * self.ngst

    def initial_state(self) -> TrackState:
        n, g = self.ncell, self.ngst
        nt = n + 2 * g
        prim = _default_prim(self.nq, nt)
        x = np.zeros(nt)
        dx = np.zeros(nt)
        X = self.xmax - self.xmin
        i = np.arange(n, dtype=np.float64)
        xc = X * (i + 0.5) / n + self.xmin
        x[g:g + n] = xc
        dx[g:g + n] = X / n
        left = xc <= self.xmid
        a = slice(g, g + n)
        prim[RHO, a] = np.where(left, self.rhoL, self.rhoR)
        prim[UU1, a] = np.where(left, self.vL, self.vR)
        prim[PPP, a] = np.where(left, self.pL, self.pR)
        prim[TR1, a] = np.where(left, self.trL, self.trR)
        xI = _prep_for_run(prim, x, dx, g)
        _update_ghosts(prim, x, dx, xI, g)
        return TrackState(nt, self.capacity, prim, x, dx, xI, np.full(nt, DT_INF), 0.0, 0)

    def resume_state(self, path: str, cfg=None) -> TrackState:
        """The -r start from a dump (Simu::reinitialise, then Simu::run's first
        updateGhosts)."""
        return _resume_1d(path, cfg or gpu.config_cart(), self.capacity, self.ngst)

    def run_params(self):
        return gpu.RunParams()


@dataclass
class Bm1dSetup:
    """1D spherical Blandford-McKee blast wave, after src/Initial/Tests/BM1D.cpp, parameterised.

    lorentz_mode 0 derives Gamma_shock^2 from tinit (BM1D.cpp LORENTZ_ == 0);
    lorentz_mode 1 takes lfac_shock2 and derives the start time (LORENTZ_ == 1).
    grid_log 0 lays ncell cells uniformly over R(1 -+ 50/Gamma_shock^2) as
    BM1D.cpp does; 1 lays them log-uniformly over [r_lo, r_hi] R."""

    n0: float = 1.0
    eta: float = 1.e-5
    Etot: float = 1.e53
    n_ext: float = 1.0
    tinit: float = 4.e6
    lfac_shock2: float = 0.0
    lorentz_mode: int = 0
    Rscale: float = 1.e17
    k: float = 0.0
    ncell: int = 9900
    nmax: int = 10000
    ngst: int = 2
    grid_log: int = 0
    r_lo: float = 0.9
    r_hi: float = 1.1
    dth: float = math.pi / 2. / 1000.
    target_ar: float = 1.0
    split_AR: float = 3.0
    merge_AR: float = 0.1
    t_bm_until: float = 1.e7
    v_in: float = 0.0
    v_out: float = 1.5
    gamma_ad: float = 4. / 3.

    nq = 10

    @property
    def capacity(self) -> int:
        return self.nmax + 2 * self.ngst

    def derived(self) -> dict:
        """BM1D.cpp:28-65 and normalizeConstants (constants.cpp:12-20)."""
        G = self.gamma_ad
        d = {}
        d["rhoNorm"] = self.n0 * MP
        d["lNorm"] = C_LIGHT
        d["vNorm"] = C_LIGHT
        d["pNorm"] = d["rhoNorm"] * d["vNorm"] * d["vNorm"]
        if self.lorentz_mode:
            d["lfacShock2"] = self.lfac_shock2
            d["tstart"] = math.pow(self.Etot * (17.) / (8. * PI * self.n_ext * MP * math.pow(C_LIGHT, 5.) *
                                                      d["lfacShock2"]), 1. / 3.)
        else:
            d["tstart"] = self.tinit
            d["lfacShock2"] = self.Etot * (17. - 4. * self.k) / (8. * PI * self.n_ext * MP *
                                                               math.pow(d["tstart"], 3) * math.pow(C_LIGHT, 5))
        d["RShock"] = C_LIGHT * d["tstart"] * (1. - 1. / (1. + 2. * (4. - self.k) * d["lfacShock2"]))
        d["rhoa"] = self.n_ext * MP * math.pow(d["RShock"] / self.Rscale, -self.k)
        d["pa"] = d["rhoa"] * self.eta * C_LIGHT * C_LIGHT
        d["ha"] = C_LIGHT * C_LIGHT + d["pa"] * G / (G - 1.) / d["rhoa"]
        d["pf"] = 2. / 3. * d["lfacShock2"] * d["ha"] * d["rhoa"]
        d["lfacf"] = math.sqrt(max(1., .5 * d["lfacShock2"]))
        d["Df"] = 2. * d["lfacShock2"] * d["rhoa"]
        d["Nalpha"] = ALPHA_SYN / (1. / (d["rhoNorm"] * d["vNorm"] * d["lNorm"]))
        d["Nmp"] = MP / (d["rhoNorm"] * math.pow(d["lNorm"], 3))
        d["Nme"] = ME / (d["rhoNorm"] * math.pow(d["lNorm"], 3))
        return d

    def run_params(self) -> "gpu.RunParams":
        d = self.derived()
        return gpu.RunParams(self.Etot, self.n_ext, self.eta, self.k, self.Rscale, d["rhoNorm"], d["pNorm"],
                             d["lNorm"], d["vNorm"], self.dth, self.target_ar, self.split_AR, self.merge_AR,
                             self.t_bm_until, self.v_in, self.v_out, d["Nalpha"], d["Nmp"], d["Nme"])

    def calc_bm(self, r_code: float, t: float):
        """Analytic BM primitives (rho, u, p) at r (code units) and t (BM1D.cpp:62-86)."""
        G, k = self.gamma_ad, self.k
        d = self.derived()
        r = r_code * d["lNorm"]
        lfacShock2 = self.Etot * (17. - 4. * k) / (8. * PI * self.n_ext * MP * math.pow(t, 3) * math.pow(C_LIGHT, 5))
        RShock = C_LIGHT * t * (1. - 1. / (1. + 2. * (4. - k) * lfacShock2))
        rhoa = self.n_ext * MP * math.pow(RShock / self.Rscale, -k)
        pa = rhoa * self.eta * C_LIGHT * C_LIGHT
        ha = C_LIGHT * C_LIGHT + pa * G / (G - 1.) / rhoa
        pf = 2. / 3. * lfacShock2 * ha * rhoa
        lfacf = math.sqrt(max(1., .5 * lfacShock2))
        Df = 2. * lfacShock2 * rhoa
        chi = (1. + 2. * (4. - k) * lfacShock2) * (1. - r / (C_LIGHT * t))
        p = pf * math.pow(chi, -(17. - 4. * k) / (12. - 3. * k)) / d["pNorm"]
        lfac = math.sqrt(lfacf * lfacf / chi + 1)
        D = Df * math.pow(chi, -(7. - 2. * k) / (4. - k))
        rho = D / lfac / d["rhoNorm"]
        u = C_LIGHT * math.sqrt(1. - 1. / (lfac * lfac)) * lfac / d["vNorm"]
        return rho, u, p

    def initial_state(self) -> TrackState:
        d = self.derived()
        n, g = self.ncell, self.ngst
        nt = n + 2 * g
        prim = _default_prim(self.nq, nt)
        x = np.zeros(nt)
        dx = np.zeros(nt)
        lNorm, RS = d["lNorm"], d["RShock"]
        if not self.grid_log:  # BM1D.cpp:100-116
            rmin = RS * (1. - 50. / d["lfacShock2"]) / lNorm
            rmax = RS * (1. + 50. / d["lfacShock2"]) / lNorm
            dr = (rmax - rmin) / n
            for i in range(n):
                x[g + i] = rmin + (i + 0.5) * dr
                dx[g + i] = dr
        else:
            rmin = self.r_lo * RS / lNorm
            rmax = self.r_hi * RS / lNorm
            lr = math.log(rmax / rmin)
            for i in range(n):
                rl = rmin * math.exp(lr * i / n)
                rr = rmin * math.exp(lr * (i + 1) / n)
                x[g + i] = 0.5 * (rl + rr)
                dx[g + i] = rr - rl
        k = self.k
        for i in range(n):  # BM1D.cpp:118-185 (one bin per cell)
            c = g + i
            r_d = x[c] * lNorm
            dr_d = dx[c] * lNorm
            if r_d > RS:
                rho = self.n_ext * MP * math.pow(r_d / self.Rscale, -k)
                prim[RHO, c] = rho / d["rhoNorm"]
                prim[UU1, c] = 0.0
                prim[PPP, c] = self.eta * rho * C_LIGHT * C_LIGHT / d["pNorm"]
                prim[TR1, c] = 1.0
            else:
                xl = r_d - dr_d / 2.
                xr = xl + dr_d
                dV = 4. / 3. * PI * (math.pow(r_d + dr_d / 2., 3) - math.pow(r_d - dr_d / 2., 3))
                xx = (xr + xl) / 2.
                ddV = 4. / 3. * PI * (xr * xr * xr - xl * xl * xl)
                chi = (1. + 2. * (4. - k) * d["lfacShock2"]) * (1. - xx / (C_LIGHT * d["tstart"]))
                dp = d["pf"] * math.pow(chi, -(17. - 4. * k) / (12. - 3. * k))
                dlfac = math.sqrt(d["lfacf"] * d["lfacf"] / chi + 1)
                dD = d["Df"] * math.pow(chi, -(7. - 2. * k) / (4. - k))
                drho = dD / dlfac
                dv = C_LIGHT * math.sqrt(1. - 1. / (dlfac * dlfac))
                rho = 0.0 + drho * ddV / dV
                v = 0.0 + dv * ddV / dV
                p = 0.0 + dp * ddV / dV
                prim[RHO, c] = rho / d["rhoNorm"]
                prim[UU1, c] = v / d["vNorm"]
                prim[PPP, c] = p / d["pNorm"]
                prim[TR1, c] = 2.0
        xI = _prep_for_run(prim, x, dx, g)
        for c in range(nt):  # radiation_initGammas
            lf = _lfac(prim[UU1, c])
            rho = prim[RHO, c]
            lim = lf * math.pow(rho, 4. / 3.)
            for q in (GMX, GMN):
                if prim[q, c] > lim / (lf * rho) or prim[q, c] <= 0.:
                    prim[q, c] = lim / (lf * rho)
        _update_ghosts(prim, x, dx, xI, g)
        t = d["tstart"]
        self._user_boundaries(prim, x, t)
        return TrackState(nt, self.capacity, prim, x, dx, xI, np.full(nt, DT_INF), t, 0)

    def _user_boundaries(self, prim, x, t):
        """userBoundaries (BM1D.cpp:254-274): the analytic BM state in the inner ghosts."""
        if t < self.t_bm_until:
            for i in range(0, self.ngst):
                rho, u, p = self.calc_bm(x[i], t)
                prim[RHO, i] = rho
                prim[UU1, i] = u
                prim[UU2, i] = 0.0
                prim[PPP, i] = p
                prim[TR1, i] = 2.0

    def resume_state(self, path: str, cfg=None) -> TrackState:
        """The -r start from a dump (Simu::reinitialise, then Simu::run's first
        updateGhosts with the BM inner boundary)."""
        st = _resume_1d(path, cfg or gpu.config_sph(gamma_ad=self.gamma_ad), self.capacity, self.ngst)
        self._user_boundaries(st.prim, st.x, st.t)
        return st


def _resume_1d(path, cfg, cap, ngst) -> TrackState:
    """gamma_text1d_read, then updateGhosts without the user hook."""
    r = gpu.text1d_read(path, cfg, cap)
    n = r["ntrack"]
    prim = np.ascontiguousarray(r["prim"][:, :n])
    x, dx = r["x"][:n].copy(), r["dx"][:n].copy()
    xI = r["xI"][:n - 1].copy()
    _update_ghosts(prim, x, dx, xI, ngst)
    return TrackState(n, cap, prim, x, dx, xI, np.full(n, DT_INF), r["t"], r["it"])


def pack(states, offsets, total, nq):
    """Pooled host arrays (the C ABI layout) from per-run TrackStates."""
    prim = np.zeros((nq, total))
    x = np.zeros(total)
    dx = np.zeros(total)
    dtl = np.full(total, DT_INF)
    xI = np.zeros(total)
    for s, o in zip(states, offsets):
        n = s.ntrack
        prim[:, o:o + n] = s.prim
        x[o:o + n] = s.x
        dx[o:o + n] = s.dx
        dtl[o:o + n] = s.dt_loc
        xI[o:o + n - 1] = s.xI
    nt = np.array([s.ntrack for s in states], dtype=np.int32)
    t = np.array([s.t for s in states])
    it = np.array([s.it for s in states], dtype=np.int64)
    return dict(ntrack=nt, t=t, it=it, prim=prim, x=x, dx=dx, dt_loc=dtl, xI=xI)


def unpack(out: dict, r: int, offsets) -> TrackState:
    """One run's TrackState from GammaGPU.download() output."""
    o = int(offsets[r])
    n = int(out["ntrack"][r])
    return TrackState(n, 0, out["prim"][:, o:o + n].copy(), out["x"][o:o + n].copy(), out["dx"][o:o + n].copy(),
                      out["xI"][o:o + n - 1].copy(), out["dt_loc"][o:o + n].copy(), float(out["t"][r]),
                      int(out["it"][r]))


@dataclass
class Jet2dSetup:
    """2D spherical (r, theta) blast wave on a wedge of theta tracks: the
    Blandford-McKee profile in the tracks whose centre lies below th_jet, cold
    ambient medium elsewhere.  The hooks follow src/Initial/Tests/BM.cpp (2D):
    uniform radial cells over [r_lo, r_hi] R_shock, LORENTZ_ == 1 start
    (Gamma_shock^2 given), ambient beyond the shock, checkCellForRegrid against
    the first active track's mean spacing, outer ghost interfaces at v_out.
    The state it builds is what Simu::initialise leaves (initialGeometry,
    initialValues, mpi_distribute, prepForRun: v2u + interfaceGeomFromCellPos,
    radiation_initGammas); the ghost tracks and cells are filled on the device
    (gamma_2d_upload with run_ghosts = 1, the updateGhosts before the loop)."""

    n0: float = 1.0
    eta: float = 1.e-10
    Etot: float = 1.e53
    n_ext: float = 1.0
    lfac_shock2: float = 2.e4
    Rscale: float = 1.e17
    k: float = 0.0
    ncell: int = 400
    ntheta: int = 16
    nmax: int = 800
    ngst: int = 2
    r_lo: float = 0.9
    r_hi: float = 1.1
    th_min: float = 0.0
    th_max: float = 0.2
    th_jet: float = 0.1
    nbins: int = 1
    split_DR: float = 5.0
    merge_DR: float = 0.3
    split_DR_slow: float = 20.0
    merge_DR_slow: float = 1.2
    v_out: float = 1.05
    it_hold: float = 1000.0
    gamma_ad: float = 4. / 3.

    nq = 10

    def derived(self) -> dict:
        """BM.cpp:13-55 (LORENTZ_ == 1) and normalizeConstants (constants.cpp:12-20)."""
        G, k = self.gamma_ad, self.k
        d = {"rhoNorm": self.n0 * MP, "lNorm": C_LIGHT, "vNorm": C_LIGHT}
        d["pNorm"] = d["rhoNorm"] * d["vNorm"] * d["vNorm"]
        d["lfacShock2"] = self.lfac_shock2
        d["tstart"] = math.pow(self.Etot * (17.) / (8. * PI * self.n_ext * MP * math.pow(C_LIGHT, 5.) *
                                                  d["lfacShock2"]), 1. / 3.)
        d["RShock"] = C_LIGHT * d["tstart"] * (1. - 1. / (1. + 2. * (4. - k) * d["lfacShock2"]))
        d["rhoa"] = self.n_ext * MP * math.pow(d["RShock"] / self.Rscale, -k)
        d["pa"] = d["rhoa"] * self.eta * C_LIGHT * C_LIGHT
        d["ha"] = C_LIGHT * C_LIGHT + d["pa"] * G / (G - 1.) / d["rhoa"]
        d["pf"] = 2. / 3. * d["lfacShock2"] * d["ha"] * d["rhoa"]
        d["lfacf"] = math.sqrt(max(1., .5 * d["lfacShock2"]))
        d["Df"] = 2. * d["lfacShock2"] * d["rhoa"]
        d["Nalpha"] = ALPHA_SYN / (1. / (d["rhoNorm"] * d["vNorm"] * d["lNorm"]))
        d["Nmp"] = MP / (d["rhoNorm"] * math.pow(d["lNorm"], 3))
        d["Nme"] = ME / (d["rhoNorm"] * math.pow(d["lNorm"], 3))
        return d

    def theta(self):
        """centre and width of each active track (BM.cpp:110-118)"""
        n = self.ntheta
        th = np.array([self.th_min + (self.th_max - self.th_min) * (j + 0.5) / n for j in range(n)])
        dth = np.full(n, (self.th_max - self.th_min) / n)
        return th, dth

    def params(self):
        from .gpu2d import Params2D
        d = self.derived()
        return Params2D(self.split_DR, self.merge_DR, self.split_DR_slow, self.merge_DR_slow, self.v_out,
                        self.it_hold, d["Nalpha"], d["Nmp"], d["Nme"])

    def _radial_profiles(self, d):
        """(r, dr, BM primitives, ambient primitives) of one track's active cells"""
        n, k = self.ncell, self.k
        lNorm, RS = d["lNorm"], d["RShock"]
        rmin = self.r_lo * RS / lNorm
        rmax = self.r_hi * RS / lNorm
        dr = (rmax - rmin) / n
        r = np.array([rmin + (i + 0.5) * dr for i in range(n)])
        bm = np.zeros((self.nq, n))
        amb = np.zeros((self.nq, n))
        for i in range(n):
            r_d, dr_d = r[i] * lNorm, dr * lNorm
            rho = self.n_ext * MP * math.pow(r_d / self.Rscale, -k)
            amb[RHO, i], amb[UU1, i], amb[PPP, i] = rho / d["rhoNorm"], 0., self.eta * rho * C_LIGHT * C_LIGHT / d["pNorm"]
            amb[TR1, i] = 1.
            if r_d > RS:
                bm[:, i] = amb[:, i]
                continue
            ddx = dr_d / self.nbins
            xl = r_d - dr_d / 2.
            xr = xl + ddx
            dV = 4. / 3. * PI * (math.pow(r_d + dr_d / 2., 3) - math.pow(r_d - dr_d / 2., 3))
            rr = v = p = 0.
            for _ in range(self.nbins):
                x = (xr + xl) / 2.
                ddV = 4. / 3. * PI * (xr * xr * xr - xl * xl * xl)
                chi = (1. + 2. * (4. - k) * d["lfacShock2"]) * (1. - x / (C_LIGHT * d["tstart"]))
                dp = d["pf"] * math.pow(chi, -(17. - 4. * k) / (12. - 3. * k))
                dlfac = math.sqrt(d["lfacf"] * d["lfacf"] / chi + 1)
                dD = d["Df"] * math.pow(chi, -(7. - 2. * k) / (4. - k))
                rr += dD / dlfac * ddV / dV
                v += C_LIGHT * math.sqrt(1. - 1. / (dlfac * dlfac)) * ddV / dV
                p += dp * ddV / dV
                xl = xr
                xr += ddx
            bm[RHO, i], bm[UU1, i], bm[PPP, i], bm[TR1, i] = rr / d["rhoNorm"], v / d["vNorm"], p / d["pNorm"], 2.
        # prepForRun: v2u (2d.cpp:1153-1172; the theta velocity is zero)
        for prof in (bm, amb):
            for i in range(n):
                vv = math.sqrt(0. + prof[UU1, i] * prof[UU1, i] + 0. * 0.)
                prof[UU1, i] *= 1. / math.sqrt(1. - vv * vv)
            # radiation_initGammas (radiation_sph.cpp:246-260)
            for i in range(n):
                u = math.sqrt(0. + prof[UU1, i] * prof[UU1, i] + 0. * 0.)
                lf = math.sqrt(1 + u * u)
                rho = prof[RHO, i]
                lim = lf * math.pow(rho, 4. / 3.)
                for q in (GMX, GMN):
                    if prof[q, i] > lim / (lf * rho) or prof[q, i] <= 0.:
                        prof[q, i] = lim / (lf * rho)
        return r, dr, bm, amb

    def initial_state(self):
        from .gpu2d import State2D
        d = self.derived()
        g, n = self.ngst, self.ncell
        NJ, cap = self.ntheta + 2 * g, self.nmax + 2 * g
        NC = NJ * cap
        r, dr, bm, amb = self._radial_profiles(d)
        prim = np.zeros((self.nq, NC))
        prim[RHO] = 1.
        prim[PPP] = 1.
        x, dx, xI = np.zeros(NC), np.zeros(NC), np.zeros(NC)
        th, _ = self.theta()
        iL = g - 1
        for jj in range(self.ntheta):
            o = (jj + g) * cap
            a = slice(o + g, o + g + n)
            prim[:, a] = bm if th[jj] <= self.th_jet else amb
            x[a], dx[a] = r, dr
            # interfaceGeomFromCellPos (2d.cpp:1055-1076): right edges, and the
            # left edge of the first active cell at index iLbnd
            xI[o + g:o + g + n] = r + dr / 2.
            xI[o + iL] = r[0] - dr / 2.
        ntrack = np.full(NJ, n + 2 * g, np.int32)
        return State2D(NJ, cap, ntrack, prim, x, dx, xI, None, None, None, None, d["tstart"], 0)
