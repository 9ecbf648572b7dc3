"""The Synge (Taub-Mathews) EOS end to end: each state's Gamma_eff in the
relativistic sound speed of the wave-speed estimates and in the shock
detector, where the reference uses GAMMA_ whatever the EOS
(gamma_config_t.eos_wavespeeds; the reference has no such switch).

The oracle is the C restatement with the same switch (oracle/gamma_oracle.c).
With the ideal EOS, Gamma_eff is GAMMA_, so the switch must change nothing.
Without the switch, the 2D step with the Synge EOS is the reference's own
(EOS_ = SYNGE_EOS_ in its environment.h), compiled as
oracle/_ref/libref_jet2d_synge.so.
"""
import multiprocessing as mp

import numpy as np
import pytest

from conftest import ref_available
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


CFG2 = dict(ncell=60, ntrack=6, nmax=120, split_DR=2.5, merge_DR=0.3, split_DR_slow=2.5, merge_DR_slow=0.3)


def _derived_synge(p):
    from oracle.refsim2d import RefJet2D
    s = RefJet2D(synge=True)
    s.set_params(**p)
    return s.derived()


def test_2d_synge_matches_reference(gpu_available):
    """The 2D wedge with the Synge EOS (Gamma = 5/3; eos_wavespeeds = 0, the
    reference's GAMMA_ in the wave speeds and the detector) against the
    reference built with EOS_ = SYNGE_EOS_ (oracle/_ref/libref_jet2d_synge.so),
    its root search converged: one step from the reference's own states after
    0, 1 and 4 steps, then 30 steps from the initial state, with identical
    cell counts; every figure is recorded beside the reference's own movement
    when only its root finder's tolerance changes (1e-15 against 4e-16).
    One step: L1 <= max(1e-11, 10x that movement), except density and u_theta
    at max(1e-9, 10x): their worst cells are the cold gas of the edge track
    (p ~ 1e-9) moving sideways at u_theta ~ 3e-7, where cons2prim's
    v = sqrt(1 - 1/lfac^2) is determined only to ~eps/v^2 ~ 1e-3 for any root
    finder; the density follows through the theta mass flux (3.7e-8 per cell
    at most, L1 5.2e-10 from the reference's step-1 state), as in the
    ideal-EOS 2D tests."""
    if not ref_available("jet2d_synge"):
        pytest.skip("oracle/_ref/libref_jet2d_synge.so not built")
    from gamma_b200 import gpu, gpu2d
    from helpers import record
    from helpers2d import l1_between_snapshots, l1_by_quantity, params_of, state_from_reference, theta_of
    from oracle.refsim2d import run_isolated
    snaps = run_isolated(CFG2, snap_at=(0, 1, 2, 4, 5, 30), c2p_epsrel=4e-16, synge=True)
    alt = run_isolated(CFG2, snap_at=(0, 1, 2, 4, 5, 30), c2p_epsrel=1e-15, synge=True)
    with mp.get_context("spawn").Pool(1) as pool:
        d = pool.apply(_derived_synge, (CFG2,))
    th, dth = theta_of(snaps[0])
    qs = (0, 1, 2, 3, 4, 6, 7)

    def run(k0, nsteps):
        g = gpu2d.Grid2DGPU(len(th), CFG2["nmax"], th, dth, gamma_ad=5. / 3., eos=gpu.EOS_SYNGE)
        g.set_params(params_of(CFG2, d))
        g.upload(state_from_reference(snaps[k0]))
        st = g.step(nsteps)
        got = g.download()
        g.close()
        ref = snaps[k0 + nsteps]
        assert st["status"] == 0 and st["c2p_fallbacks"] == 0
        assert [int(got.ntrack[j]) for j in range(len(ref.tracks))] == [t.ntrack for t in ref.tracks]
        return got, ref

    for k in (0, 1, 4):
        got, ref = run(k, 1)
        assert abs(got.t - ref.t) <= 1e-14 * ref.t, k
        l1 = l1_by_quantity(got, ref, qs=qs)
        self_l1 = l1_between_snapshots(alt[k + 1], ref, qs)
        # rho and u_theta: the slow cold cells at the wedge edge (see above)
        bar = {q: max(1e-9 if q in (0, 3) else 1e-11, 10 * self_l1[q]) for q in qs}
        for q in qs:
            record(f"one step from step {k}: L1 slot {q} (reference tolerance sensitivity {self_l1[q]:.2e})",
                   l1[q], bar[q])
        assert all(l1[q] <= bar[q] for q in qs), (k, l1, self_l1)
    got, ref = run(0, 30)
    assert abs(got.t - ref.t) <= 1e-10 * ref.t
    l1 = l1_by_quantity(got, ref, qs=qs)
    self_l1 = l1_between_snapshots(alt[30], ref, qs)
    bar = {q: 1e-6 if q == 3 else 3e-8 for q in qs}
    for q in qs:
        record(f"30 steps L1 slot {q} (reference tolerance sensitivity {self_l1[q]:.2e})", l1[q], bar[q])
    assert all(l1[q] <= bar[q] for q in qs), (l1, self_l1)
