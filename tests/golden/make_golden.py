"""Writes the golden fixtures of this directory from the GAMMA reference itself.

The reference is the one compiled from its sources by oracle/Makefile
(oracle/_ref/libref_*.so; the checkout is $GAMMA_REFERENCE, else the directory
"reference" beside this repository).  Each fixture holds the reference's
track state at a few steps of a small case, so that the oracle restatement and
the GPU path can be pinned on machines without the reference sources:

  tube.npz       planar shock tube (300 cells), steps 0, 1, 5
  bm1d.npz       BM1D blast wave (300 log cells), steps 0, 1, 10
  jet2d.npz      2D wedge (4 theta tracks of 48 cells), steps 0 and 3, with the
                 root search converged (the smoke check's case)

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

TUBE = dict(ncell=300, nmax=300, vL=0.3, vR=0.3, rhoL=11., pL=12.)
BM1D = dict(eta=1e-8, lorentz_mode=1, lfac_shock2=400., ncell=300, nmax=600, grid_log=1, r_lo=0.97, r_hi=1.03)
JET = dict(ncell=48, ntrack=4, nmax=96, split_DR=2.5, merge_DR=0.3, split_DR_slow=2.5, merge_DR_slow=0.3)
FIELDS = ("prim", "x", "dx", "dt_loc", "sd", "shocked", "xI")


def one_d(kind, params, steps, name):
    from oracle.refsim import run_isolated
    snaps = run_isolated(kind, params, max(steps), snap_at=steps)
    out = {"steps": np.array(steps), "params": np.array(repr(params))}
    for k in steps:
        s = snaps[k]
        out[f"s{k}_scalars"] = np.array([s.t, s.dt, s.it, s.ntrack])
        for f in FIELDS:
            out[f"s{k}_{f}"] = getattr(s, f)
    np.savez_compressed(os.path.join(HERE, name), **out)


def two_d(params, steps, name, epsrel):
    from oracle.refsim2d import run_isolated
    snaps = run_isolated(params, snap_at=steps, c2p_epsrel=epsrel)
    out = {"steps": np.array(steps), "params": np.array(repr(params)), "epsrel": np.array(epsrel)}
    for k in steps:
        g = snaps[k]
        out[f"s{k}_scalars"] = np.array([g.t, g.dt, g.it, g.cap])
        for j, t in enumerate(g.tracks):
            out[f"s{k}_j{j}_n"] = np.array(t.ntrack)
            for f in ("prim", "x", "dx", "th", "dth", "xI"):
                out[f"s{k}_j{j}_{f}"] = getattr(t, f)
        out[f"s{k}_ntracks"] = np.array(len(g.tracks))
    np.savez_compressed(os.path.join(HERE, name), **out)


if __name__ == "__main__":
    one_d("tube", TUBE, (0, 1, 5), "tube.npz")
    one_d("bm1d", BM1D, (0, 1, 10), "bm1d.npz")
    two_d(JET, (0, 3), "jet2d.npz", 4e-16)
    print("written:", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))
