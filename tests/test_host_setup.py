"""Host-side problem set-up (gamma_b200.problems) against the oracle's initialisation."""
import numpy as np
import pytest

from gamma_b200 import problems
from oracle import port


def _same(s, snap):
    assert s.ntrack == snap.ntrack
    for f in ("prim", "x", "dx", "dt_loc", "xI"):
        assert np.array_equal(getattr(s, f), getattr(snap, f)), f
    assert s.t == snap.t


@pytest.mark.parametrize("kw", [dict(ncell=500, vL=0.3, vR=0.3, rhoL=11., pL=12.), dict(ncell=257, xmid=0.4)])
def test_tube_initial_state(kw):
    ps = port.PortSim(port.tube_config(nmax=kw["ncell"], **kw))
    ps.init()
    _same(problems.TubeSetup(**kw).initial_state(), ps.snapshot())


@pytest.mark.parametrize("kw", [dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, ncell=2000, nmax=4000, grid_log=1),
                                dict(ncell=900, nmax=1000)])
def test_bm1d_initial_state(kw):
    ps = port.PortSim(port.bm1d_config(**kw))
    ps.init()
    _same(problems.Bm1dSetup(**kw).initial_state(), ps.snapshot())


def test_bm1d_run_params_match_oracle_constants():
    kw = dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, ncell=2000, nmax=4000, grid_log=1)
    ps = port.PortSim(port.bm1d_config(**kw))
    sc = ps.scalars()
    rp = problems.Bm1dSetup(**kw).run_params()
    assert rp.Nalpha == sc["Nalpha"] and rp.Nmp == sc["Nmp"] and rp.Nme == sc["Nme"]
    assert rp.rhoNorm == sc["rhoNorm"] and rp.pNorm == sc["pNorm"]


def test_pack_unpack_roundtrip():
    states = [problems.TubeSetup(ncell=n).initial_state() for n in (10, 33, 64)]
    offs = np.array([0, 16, 54])
    packed = problems.pack(states, offs, 128, 6)
    out = dict(packed, dt=np.zeros(3), status=np.zeros(3))
    for r, s in enumerate(states):
        u = problems.unpack(out, r, offs)
        assert np.array_equal(u.prim, s.prim) and np.array_equal(u.xI, s.xI)
