"""The 2D initial state built on the host equals the reference's (Simu::initialise
of the NUM_D = 2 build with the theta-wedge blast-wave module) bit for bit."""
import multiprocessing as mp

import numpy as np
import pytest

from conftest import ref_available


def _ref_init(p):
    from oracle.refsim2d import RefJet2D
    s = RefJet2D()
    s.set_params(**p)
    s.init()
    return s.snapshot()


@pytest.mark.parametrize("nbins", [1, 7])
def test_jet2d_initial_state_matches_reference(nbins):
    if not ref_available("jet2d"):
        pytest.skip("oracle/_ref/libref_jet2d.so not built")
    from gamma_b200 import problems
    setup = problems.Jet2dSetup(ncell=120, ntheta=7, nmax=200, nbins=nbins, th_jet=0.1)
    p = dict(ncell=120, ntrack=7, nmax=200, nbins=nbins, th_jet=0.1)
    with mp.get_context("spawn").Pool(1) as pool:
        ref = pool.apply(_ref_init, (p,))
    st = setup.initial_state()
    th, dth = setup.theta()
    assert st.t == ref.t and ref.cap == st.cap
    g = setup.ngst
    for jj in range(setup.ntheta):
        j = jj + g
        b = ref.tracks[j]
        assert b.ntrack == st.ntrack[j]
        assert b.th[g] == th[jj] and b.dth[g] == dth[jj]
        a = st.track(j)
        s = slice(g, b.ntrack - g)
        assert np.array_equal(a["prim"][:, s], b.prim[:, s])
        assert np.array_equal(a["x"][s], b.x[s]) and np.array_equal(a["dx"][s], b.dx[s])
        # interfaces iLbnd .. iRbnd-1 (the rest are ghost interfaces)
        assert np.array_equal(a["xI"][g - 1:b.ntrack - g], b.xI[g - 1:b.ntrack - g])
