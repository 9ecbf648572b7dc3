"""The oracle restatement (oracle/gamma_oracle.c) against the reference itself.

The reference sources, compiled unmodified with a one-rank MPI header and a
Brent root finder behind the GSL names (oracle/_ref), and the C restatement
must agree bit for bit on every field of the track, step after step.  The only
field excluded is the spectral-index candidate of cells that are not shocked:
there the reference reads an uninitialised local (src/Radiation/radiation_sph.cpp:162,
left unset when compute_Sd returns early at :56-57), and the value never
reaches the solution (it is used only for shocked cells, :271-272).
"""
import numpy as np
import pytest

from conftest import ref_available
from oracle import port
from oracle.refsim import run_isolated

FIELDS = ("prim", "x", "dx", "dt_loc", "sd", "shocked", "xI")


def assert_same(a, b, label):
    assert a.ntrack == b.ntrack, f"{label}: ntrack {a.ntrack} != {b.ntrack}"
    assert a.t == b.t and a.dt == b.dt, f"{label}: t/dt differ"
    for f in FIELDS:
        A, B = getattr(a, f), getattr(b, f)
        assert np.array_equal(A, B, equal_nan=True), f"{label}: field {f} differs"
    ps_a = np.where(a.shocked > 0, a.pspec, 0.0)
    ps_b = np.where(b.shocked > 0, b.pspec, 0.0)
    assert np.array_equal(ps_a, ps_b), f"{label}: pspec of shocked cells differs"


def port_run(cfg, steps):
    s = port.PortSim(cfg)
    s.init()
    out = {0: s.snapshot()}
    done = 0
    for k in sorted(steps):
        s.step(k - done)
        done = k
        out[k] = s.snapshot()
    return out


CASES = {
    "tube": ("tube", dict(ncell=300, nmax=300, vL=0.3, vR=0.3, rhoL=11., pL=12.), (1, 5, 40)),
    "tube_fast": ("tube", dict(ncell=200, nmax=200, vL=-0.45, vR=-0.45, rhoL=8.7, pL=15.1), (1, 30)),
    "bm1d_log_g100": ("bm1d", dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, ncell=2000, nmax=4000,
                                   grid_log=1), (1, 2, 25, 100)),
    "bm1d_small": ("bm1d", dict(eta=1e-8, lorentz_mode=1, lfac_shock2=400., ncell=300, nmax=600, grid_log=1,
                                r_lo=0.97, r_hi=1.03), (1, 10, 60)),
    # the Euler time-stepping module (Timestep/euler.cpp linked in place of rk3.cpp)
    "tube_euler": ("tube_euler", dict(ncell=300, nmax=300, vL=0.3, vR=0.3, rhoL=11., pL=12.), (1, 5, 60)),
    "bm1d_small_euler": ("bm1d_euler", dict(eta=1e-8, lorentz_mode=1, lfac_shock2=400., ncell=300, nmax=600,
                                            grid_log=1, r_lo=0.97, r_hi=1.03), (1, 10, 60)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_restatement_matches_reference(name):
    kind, params, steps = CASES[name]
    if not ref_available(kind):
        pytest.skip("reference build oracle/_ref absent")
    ref = run_isolated(kind, params, max(steps), snap_at=(0,) + steps)
    ts = 1 if kind.endswith("_euler") else 0
    cfg = port.tube_config(timestep=ts, **params) if kind.startswith("tube") else port.bm1d_config(timestep=ts, **params)
    mine = port_run(cfg, steps)
    for k in (0,) + steps:
        assert_same(mine[k], ref[k], f"{name} step {k}")


@pytest.mark.slow
def test_restatement_matches_reference_bm1d_original():
    """The reference's own Tests/BM1D.cpp (9900 uniform cells, eta 1e-5), unmodified."""
    if not ref_available("bm1d_orig"):
        pytest.skip("reference build oracle/_ref absent")
    ref = run_isolated("bm1d_orig", {}, 2, snap_at=(0, 1, 2))
    mine = port_run(port.bm1d_config(), (1, 2))
    for k in (0, 1, 2):
        assert_same(mine[k], ref[k], f"bm1d_orig step {k}")
