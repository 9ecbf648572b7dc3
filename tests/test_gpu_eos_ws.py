"""The Synge (Taub-Mathews) EOS end to end: each state's Gamma_eff in the
relativistic sound speed of the wave-speed estimates and in the shock
detector, where the reference uses GAMMA_ whatever the EOS
(gamma_config_t.eos_wavespeeds; the reference has no such switch).

The oracle is the C restatement with the same switch (oracle/gamma_oracle.c).
With the ideal EOS, Gamma_eff is GAMMA_, so the switch must change nothing.
"""
import numpy as np
import pytest

from helpers import l1_rel

pytestmark = pytest.mark.gpu

KW = dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, ncell=400, nmax=800, grid_log=1, r_lo=0.98, r_hi=1.02)


def _bm1d(cfg, setup, nsteps):
    from gamma_b200 import gpu, problems
    g = gpu.GammaGPU(cfg, [setup.capacity])
    g.set_params([setup.run_params()])
    pk = problems.pack([setup.initial_state()], g.offsets, g.total, 10)
    g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])
    st = g.step(nsteps)
    out = problems.unpack(g.download(), 0, g.offsets)
    g.close()
    return st, out


def _jet(eos, gamma_ad, ws, nsteps):
    from gamma_b200 import gpu2d, problems
    s = problems.Jet2dSetup(ncell=100, ntheta=6, nmax=200, split_DR=2.5, merge_DR=0.3, split_DR_slow=2.5,
                            merge_DR_slow=0.3)
    th, dth = s.theta()
    g = gpu2d.Grid2DGPU(s.ntheta, s.nmax, th, dth, gamma_ad=gamma_ad, eos=eos, eos_wavespeeds=ws)
    g.set_params(s.params())
    g.upload(s.initial_state(), run_ghosts=True)
    st = g.step(nsteps)
    out = g.download()
    g.close()
    return st, out


def test_switch_changes_nothing_with_the_ideal_eos(gpu_available):
    from gamma_b200 import gpu, problems
    setup = problems.Bm1dSetup(**KW)
    _, a = _bm1d(gpu.config_sph(), setup, 30)
    _, b = _bm1d(gpu.config_sph(eos_wavespeeds=1), setup, 30)
    assert a.ntrack == b.ntrack
    assert np.array_equal(a.prim, b.prim) and np.array_equal(a.x, b.x) and np.array_equal(a.xI, b.xI)
    _, a2 = _jet(gpu.EOS_IDEAL, 4. / 3., 0, 8)
    _, b2 = _jet(gpu.EOS_IDEAL, 4. / 3., 1, 8)
    assert np.array_equal(a2.ntrack, b2.ntrack)
    for j in range(a2.NJ):
        o, n = j * a2.cap, int(a2.ntrack[j])
        assert np.array_equal(a2.prim[:, o:o + n], b2.prim[:, o:o + n]), j


def test_synge_end_to_end_matches_oracle(gpu_available):
    """BM1D blast wave with the Synge EOS (Gamma = 5/3) and Gamma_eff in the
    wave speeds and the detector, against the C restatement with the same
    switch: identical cell counts and L1 <= 1e-8 after 40 steps.  The switch
    moves the solution well beyond that bar, so the test sees it."""
    from gamma_b200 import gpu, problems
    from oracle import port
    kw = dict(KW, gamma_ad=5. / 3.)
    setup = problems.Bm1dSetup(**kw)
    ps = port.PortSim(port.bm1d_config(c2p_epsrel=1e-15, eos=1, eos_wavespeeds=1, **kw))
    ps.init()
    init = ps.snapshot()
    st0 = setup.initial_state()
    assert init.ntrack == st0.ntrack and np.array_equal(init.x, st0.x)
    assert np.array_equal(init.prim[:, 2:-2], st0.prim[:, 2:-2])
    ps.step(40)
    ref = ps.snapshot()
    st, got = _bm1d(gpu.config_sph(gamma_ad=5. / 3., eos=gpu.EOS_SYNGE, eos_wavespeeds=1), setup, 40)
    assert st["status"] == 0 and st["c2p_fallbacks"] == 0
    assert got.ntrack == ref.ntrack
    a = slice(2, got.ntrack - 2)
    for q in (0, 1, 2, 4, 6, 7):
        assert l1_rel(got.prim[q, a], ref.prim[q, a]) <= 1e-8, q
    _, off = _bm1d(gpu.config_sph(gamma_ad=5. / 3., eos=gpu.EOS_SYNGE), setup, 40)
    if off.ntrack == got.ntrack:
        moved = max(l1_rel(off.prim[q, a], got.prim[q, a]) for q in (0, 1, 2))
    else:
        moved = 1.
    assert moved > 1e-6, moved


def test_2d_synge_end_to_end_runs(gpu_available):
    """The 2D wedge with the Synge EOS and the switch: no fallback, finite
    states, and a solution that the switch moves."""
    from gamma_b200 import gpu
    st, a = _jet(gpu.EOS_SYNGE, 5. / 3., 1, 10)
    assert st["status"] == 0 and st["c2p_fallbacks"] == 0
    _, b = _jet(gpu.EOS_SYNGE, 5. / 3., 0, 10)
    num = den = 0.
    for j in range(2, a.NJ - 2):
        o, n = j * a.cap, int(a.ntrack[j])
        assert np.all(np.isfinite(a.prim[:, o:o + n])), j
        if int(b.ntrack[j]) == n:
            num += np.sum(np.abs(a.prim[1, o + 2:o + n - 2] - b.prim[1, o + 2:o + n - 2]))
            den += np.sum(np.abs(b.prim[1, o + 2:o + n - 2]))
    assert num / den > 1e-8
