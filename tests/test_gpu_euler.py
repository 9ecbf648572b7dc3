"""The Euler time-stepping module (src/Timestep/euler.cpp): Grid::evolve is
one Grid::update, so a step is the first RK3 stage alone, followed by the
particle injection.  The cells the update does not move (every ghost,
including cells iLbnd and iRbnd) keep the geometry of their stage-1 copies.

1D runs are compared with the C restatement run with timestep = 1, which is
pinned bit for bit to the reference built with euler.cpp in place of rk3.cpp
(tests/test_oracle_pin.py); the 2D run is compared with that 2D build itself
(oracle/_ref/libref_jet2d_euler.so).  The 1D tolerances are those of the RK3
parity tests (test_gpu_parity.py), which explain them; the 2D test explains its
own.
"""
import multiprocessing as mp

import numpy as np
import pytest

from conftest import ref_available
from helpers import l1_rel, record
from helpers2d import l1_between_snapshots, l1_by_quantity, params_of, state_from_reference, theta_of

pytestmark = pytest.mark.gpu

TUBES = [(64, 0.0, 10.0, 13.33), (300, -0.45, 8.5, 15.0), (1000, 0.49, 12.0, 10.7)]
BM_SMALL = dict(eta=1e-8, lorentz_mode=1, lfac_shock2=400., ncell=300, nmax=600, grid_log=1, r_lo=0.97, r_hi=1.03)
BM_CFG0 = dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, ncell=2000, nmax=4000, grid_log=1)


def _tubes_gpu(setups, nsteps, timestep):
    from gamma_b200 import gpu, problems
    g = gpu.GammaGPU(gpu.config_cart(timestep=timestep), [s.capacity for s in setups])
    pk = problems.pack([s.initial_state() for s in setups], g.offsets, g.total, 6)
    g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])
    st = g.step(nsteps)
    out = [problems.unpack(g.download(), r, g.offsets) for r in range(len(setups))]
    g.close()
    return out, st


def _tube_port(s, nsteps, epsrel=1e-13):
    from oracle import port
    ps = port.PortSim(port.tube_config(ncell=s.ncell, nmax=s.ncell, xmin=s.xmin, xmax=s.xmax, xmid=s.xmid,
                                       rhoL=s.rhoL, pL=s.pL, vL=s.vL, trL=s.trL, rhoR=s.rhoR, pR=s.pR, vR=s.vR,
                                       trR=s.trR, timestep=1, c2p_epsrel=epsrel))
    ps.init()
    ps.step(nsteps)
    return ps.snapshot()


def _geometry_close(got, ref, rtol):
    for f in ("x", "dx", "xI"):  # ghosts included: their stage-1 copies
        a, b = getattr(got, f), getattr(ref, f)
        assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)) <= rtol, f


def test_euler_tubes_match_oracle(gpu_available):
    from gamma_b200 import problems
    setups = [problems.TubeSetup(ncell=n, vL=v, vR=v, rhoL=r, pL=p) for n, v, r, p in TUBES]
    one, st = _tubes_gpu(setups, 1, 1)
    assert st["status"] == 0
    for s, g in zip(setups, one):
        ref = _tube_port(s, 1, epsrel=1e-16)  # converged root search
        assert g.ntrack == ref.ntrack
        _geometry_close(g, ref, 1e-12)
        a = slice(2, g.ntrack - 2)
        for q in (0, 1, 2, 4):
            assert l1_rel(g.prim[q, a], ref.prim[q, a]) <= 1e-11, q
        assert abs(g.t - ref.t) <= 1e-14 * abs(ref.t)
    many, st = _tubes_gpu(setups, 150, 1)
    assert st["status"] == 0 and st["c2p_fallbacks"] == 0
    rk3, _ = _tubes_gpu(setups, 150, 0)
    for s, g, h in zip(setups, many, rk3):
        ref = _tube_port(s, 150)
        a = slice(2, g.ntrack - 2)
        for q in (0, 1, 2, 4):
            assert l1_rel(g.prim[q, a], ref.prim[q, a]) <= 1e-8, q
        assert l1_rel(g.xI, ref.xI) <= 1e-8
        assert abs(g.t - ref.t) <= 1e-10 * abs(ref.t)
        # the switch is live: RK3 lands elsewhere
        assert l1_rel(h.prim[0, a], g.prim[0, a]) > 1e-6


def _bm_gpu(kw, timestep):
    from gamma_b200 import gpu, problems
    s = problems.Bm1dSetup(**kw)
    g = gpu.GammaGPU(gpu.config_sph(timestep=timestep), [s.capacity])
    g.set_params([s.run_params()])
    pk = problems.pack([s.initial_state()], g.offsets, g.total, 10)
    g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])
    return g


@pytest.mark.parametrize("kw", [BM_SMALL, BM_CFG0], ids=["bm1d_small", "bm1d_g100"])
def test_euler_bm1d_matches_oracle(gpu_available, kw):
    """BM1D with regrid, shock detection and synchrotron: identical cell counts,
    regrid actions and ghost geometry, L1 <= 1e-8 over 300 steps."""
    from gamma_b200 import problems
    from oracle import port
    g = _bm_gpu(kw, 1)
    ps = port.PortSim(port.bm1d_config(timestep=1, **kw))
    ps.init()
    for chunk in (1, 29, 270):
        st = g.step(chunk)
        assert st["status"] == 0 and st["c2p_fallbacks"] == 0
        ps.step(chunk)
        got = problems.unpack(g.download(), 0, g.offsets)
        ref = ps.snapshot()
        assert got.ntrack == ref.ntrack, (chunk, got.ntrack, ref.ntrack)
        a = slice(2, got.ntrack - 2)
        for q in (0, 1, 2, 4, 6, 7):
            assert l1_rel(got.prim[q, a], ref.prim[q, a]) <= 1e-8, (chunk, q)
        assert np.max(np.abs(got.x - ref.x) / np.abs(ref.x)) <= 1e-10
        assert np.max(np.abs(got.dx - ref.dx) / np.abs(ref.x)) <= 1e-10
        assert abs(got.t - ref.t) <= 1e-12 * ref.t
    g.close()


CFG2 = dict(ncell=60, ntrack=6, nmax=120, split_DR=2.5, merge_DR=0.3, split_DR_slow=2.5, merge_DR_slow=0.3)


def _derived(p):
    from oracle.refsim2d import RefJet2D
    s = RefJet2D()
    s.set_params(**p)
    return s.derived()


def test_euler_2d_matches_reference(gpu_available):
    """The 2D wedge with the reference built with euler.cpp.

    One step from the reference's own states (steps 0, 1 and 4, with the
    fields it carries between steps) agrees at L1 <= 1e-12 (measured <= 1e-13)
    and 1e-12 per cell in density, ghost-copy geometry of cells iLbnd and
    iRbnd included.

    Over 30 steps from the initial state the agreement is looser, because this
    problem amplifies last-bit differences: the GPU's Newton and the
    reference's Brent leave different last bits in the pressure root of about
    half the cells, and the cold ambient gas (p/rho ~ 1e-10, where the pressure
    comes out of a cancellation in tau) grows them step by step.  The reference
    itself, compiled with FMA contraction, differs from its plain build by L1 ~1e-4
    in density after 30 steps.  The bars are L1 <= 3e-8 (1e-6 for u_theta, ~0
    away from the jet edge), with identical cell counts and t within 1e-10;
    measured 7.9e-9 (rho), 1.1e-8 (p), 5.5e-9 (u_r), 3.8e-7 (u_theta),
    1.6e-8 (gamma_min tracer).  The reference's movement when only its root
    finder's tolerance changes (1e-15 against 4e-16) is recorded beside each
    figure (2.9e-9 in rho, 1e-10 in u_theta): it does not measure which point
    of the cold cells' flat f(p) band a second root finder stops at."""
    if not ref_available("jet2d_euler"):
        pytest.skip("oracle/_ref/libref_jet2d_euler.so not built")
    from gamma_b200 import gpu, gpu2d
    from oracle.refsim2d import run_isolated
    snaps = run_isolated(CFG2, snap_at=(0, 1, 2, 4, 5, 30), c2p_epsrel=4e-16, euler=True)
    alt = run_isolated(CFG2, snap_at=(30,), c2p_epsrel=1e-15, euler=True)
    with mp.get_context("spawn").Pool(1) as pool:
        d = pool.apply(_derived, (CFG2,))
    th, dth = theta_of(snaps[0])

    def run(k0, nsteps):
        g = gpu2d.Grid2DGPU(len(th), CFG2["nmax"], th, dth, timestep=gpu.TS_EULER)
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
        l1 = l1_by_quantity(got, ref)
        assert all(v <= 1e-12 for v in l1.values()), (k, l1)
        for j in range(2, len(ref.tracks) - 2):
            a, b = got.track(j), ref.tracks[j]
            s = slice(1, b.ntrack - 1)  # cells iLbnd and iRbnd keep their ghost copies
            assert np.max(np.abs(a["x"][s] - b.x[s]) / b.x[s]) <= 1e-12, (k, j)
            assert np.max(np.abs(a["dx"][s] - b.dx[s]) / b.x[s]) <= 1e-12, (k, j)
            assert np.max(np.abs(a["xI"] - b.xI) / b.xI) <= 1e-12, (k, j)
            a0 = slice(2, b.ntrack - 2)
            assert np.max(np.abs(a["prim"][0][a0] - b.prim[0][a0]) / b.prim[0][a0]) <= 1e-12, (k, j)
    got, ref = run(0, 30)
    assert abs(got.t - ref.t) <= 1e-10 * ref.t
    l1 = l1_by_quantity(got, ref)
    self_l1 = l1_between_snapshots(alt[30], ref, tuple(l1))
    bar = {q: 1e-6 if q == 3 else 3e-8 for q in l1}
    for q, v in l1.items():
        record(f"30 steps L1 slot {q} (reference tolerance sensitivity {self_l1[q]:.2e})", v, bar[q])
    assert all(v <= bar[q] for q, v in l1.items()), (l1, self_l1)
