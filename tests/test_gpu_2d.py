"""Parity of the 2D (r, theta) CUDA step with the GAMMA reference built with NUM_D = 2.

The reference (oracle/_ref/libref_jet2d.so: the reference's own 2d.cpp,
spherical.cpp, rel_sph.cpp, rk3.cpp, radiation_sph.cpp, with a theta-wedge
blast-wave problem module) is the oracle here.  Runs start from the
reference's own snapshots -- including the fields it carries between stages
(gradients, neighbour lists, dt_loc) -- so one GPU step is compared with one
reference step.

Tolerances.  The reference runs with its cons2prim root search converged (the
Brent stopping tolerance set to 4e-16 instead of 1e-13 through the GSL shim).
Its own result moves by L1 ~5e-9 (density) over 30 steps when only that
tolerance changes, because slow cells amplify rounding: the velocity of a cell
comes from v = sqrt(1 - 1/lfac^2), whose relative error is ~eps/v^2, and the
density follows through the fluxes.  Hence per-cell checks keep a share of
cells (most within 1e-12) and global L1 bars: <= 1e-9 after one step,
<= 1e-8 after 30 steps.  Cell counts, regrid decisions and neighbour lists are
compared exactly.
"""
import multiprocessing as mp

import numpy as np
import pytest

from conftest import ref_available
from helpers import record
from helpers2d import cell_errors, l1_between_snapshots, l1_by_quantity, params_of, state_from_reference, theta_of

pytestmark = pytest.mark.gpu

CFG = dict(ncell=60, ntrack=6, nmax=120, split_DR=2.5, merge_DR=0.3, split_DR_slow=2.5, merge_DR_slow=0.3)
EPS_CONVERGED = 4e-16


def _derived(p):
    from oracle.refsim2d import RefJet2D
    s = RefJet2D()
    s.set_params(**p)
    return s.derived()


@pytest.fixture(scope="module")
def ref2d():
    if not ref_available("jet2d"):
        pytest.skip("oracle/_ref/libref_jet2d.so not built")
    from oracle.refsim2d import run_isolated
    snaps = run_isolated(CFG, snap_at=(0, 1, 3, 4, 30), c2p_epsrel=EPS_CONVERGED)
    with mp.get_context("spawn").Pool(1) as pool:
        d = pool.apply(_derived, (CFG,))
    return snaps, d


def _gpu(snaps, d):
    from gamma_b200 import gpu2d
    th, dth = theta_of(snaps[0])
    g = gpu2d.Grid2DGPU(len(th), CFG["nmax"], th, dth)
    g.set_params(params_of(CFG, d))
    return g


def _same_counts(got, ref):
    return [int(got.ntrack[j]) for j in range(len(ref.tracks))] == [t.ntrack for t in ref.tracks]


@pytest.mark.parametrize("k", [0, 3])
def test_2d_one_step_matches_reference(gpu_available, ref2d, k):
    snaps, d = ref2d
    g = _gpu(snaps, d)
    g.upload(state_from_reference(snaps[k]))
    st = g.step(1)
    got = g.download()
    ref = snaps[k + 1]
    g.close()
    assert st["status"] == 0
    assert _same_counts(got, ref)
    assert abs(got.t - ref.t) <= 1e-14 * ref.t
    for j in range(2, len(ref.tracks) - 2):
        a, b = got.track(j), ref.tracks[j]
        s = slice(2, b.ntrack - 2)
        # interface speeds are lambda*, which cold gas conditions poorly
        assert np.max(np.abs(a["x"][s] - b.x[s]) / b.x[s]) <= 1e-11
        assert np.max(np.abs(a["dx"][s] - b.dx[s]) / b.x[s]) <= 1e-11
        assert np.max(np.abs(a["xI"] - b.xI) / b.xI) <= 1e-11
    l1 = l1_by_quantity(got, ref)
    assert all(v <= 1e-9 for v in l1.values()), l1
    # the reference's own one-step result moves by up to ~4e-9 in slow cells
    # when only its root finder's tolerance changes
    for q in (0, 1, 4, 6, 7):
        e = cell_errors(got, ref, q)
        assert np.mean(e <= 1e-12) >= 0.9, (q, np.mean(e <= 1e-12))
        assert np.max(e) <= 1e-8, (q, np.max(e))


def test_2d_30_steps_l1(gpu_available, ref2d):
    snaps, d = ref2d
    g = _gpu(snaps, d)
    g.upload(state_from_reference(snaps[0]))
    st = g.step(30)
    got = g.download()
    g.close()
    ref = snaps[30]
    assert st["status"] == 0 and st["c2p_fallbacks"] == 0
    assert _same_counts(got, ref)
    assert abs(got.t - ref.t) <= 1e-11 * ref.t
    l1 = l1_by_quantity(got, ref)
    assert all(v <= 1e-8 for v in l1.values()), l1


def _ref_prepared(args):
    p, k = args
    from oracle.refsim2d import RefJet2D
    s = RefJet2D()
    s.set_params(**p)
    s.init()
    s.set_c2p_epsrel(EPS_CONVERGED)
    if k:
        s.step(k)
    before = s.snapshot()
    s.partial(2)
    after = s.snapshot()
    return before, after, [s.fluxes(j, after.cap) for j in range(len(after.tracks))]


@pytest.mark.parametrize("k", [0, 3])
def test_2d_stage1_fluxes_match_reference(gpu_available, ref2d, k):
    """From the same state, regrid + ghosts + the stage-1 flux pass give the
    reference's neighbour lists, grad_mv, this stage's grad_f1, interface
    speeds and all fluxes: no root finder is involved up to this point."""
    snaps, d = ref2d
    with mp.get_context("spawn").Pool(1) as pool:
        before, after, fl = pool.apply(_ref_prepared, ((CFG, k),))
    g = _gpu(snaps, d)
    g.upload(state_from_reference(before))
    g.prepare()
    got = g.download()
    f = g.download_fluxes()
    g.close()
    assert _same_counts(got, after)
    cap = got.cap

    def rel(a, b):
        scale = max(np.max(np.abs(b)), 1e-300)
        return float(np.max(np.abs(a - b)) / scale) if b.size else 0.

    for j, b in enumerate(after.tracks):
        o, n = j * cap, b.ntrack
        cf, itf = fl[j]
        for side in (0, 1):  # neighbour lists (first id only where the list is not empty)
            cnt = got.nbr[2 * side + 1, o:o + n]
            assert np.array_equal(cnt, b.nbr[:, side, 1]), (j, side)
            has = cnt > 0
            assert np.array_equal(got.nbr[2 * side, o:o + n][has], b.nbr[has, side, 0]), (j, side)
        assert rel(f["v"][o:o + n - 1], itf[0]) <= 1e-14, j
        assert rel(f["lL"][o:o + n - 1], itf[1]) <= 1e-14, j
        assert rel(f["lR"][o:o + n - 1], itf[2]) <= 1e-14, j
        for q in range(10):
            assert rel(f["flux"][q, o:o + n - 1], itf[3 + q]) <= 1e-13, (j, q)
            assert rel(f["f1lo"][q, o:o + n], cf[0, 1, q]) <= 1e-13, (j, q)
            assert rel(f["f1hi"][q, o:o + n], cf[1, 1, q]) <= 1e-13, (j, q)
            assert rel(got.grad_mv[q, o:o + n], b.grad_mv[q]) <= 1e-13, (j, q)
            if j < len(after.tracks) - 1:  # the last track keeps its copied value
                gr, gf = f["grad_f1"][q, o:o + n], b.grad_f1[q]
                ok = np.isfinite(gf)  # cells without neighbours: 0/0 in both
                assert np.array_equal(np.isfinite(gr), ok), (j, q)
                assert rel(gr[ok], gf[ok]) <= 1e-13, (j, q)
        assert np.max(np.abs(got.extra["sd"][o:o + n] - b.sd)) <= 1e-12, j
        assert np.array_equal(got.dt_loc[o:o + n] == b.dt_loc, np.ones(n, bool)) or \
            rel(got.dt_loc[o:o + n], b.dt_loc) <= 1e-14, j


def _ref_after_regrid(p):
    from oracle.refsim2d import RefJet2D
    s = RefJet2D()
    s.set_params(**p)
    s.init()
    s.set_c2p_epsrel(EPS_CONVERGED)
    before = s.snapshot()
    s.partial(1)
    return before, s.snapshot()


def test_2d_heavy_regrid_matches_reference(gpu_available):
    """The reference problem module's own ratios (merge below 1.2x the target
    spacing where lfac < 2) merge about two thirds of the cells in the first
    step.  The regrid itself is compared exactly: cell counts, positions,
    widths and interfaces, and the merged states within rounding (a merged
    cold cell's pressure is a root of f(p) that is flat to within eps*E there,
    so the two root finders settle at different points of that band: 1e-10
    against 1.00000008e-10).  That difference then reaches the shock front, so
    the steps after it are held to L1 <= 1e-7 (1e-6 for the synchrotron
    tracers, which are re-injected wherever the shock detector fires); measured
    9.4e-9 (rho), 2.3e-8 (p), 1.6e-8 (u_r) after one step.  The reference's own
    movement when only its root finder's tolerance changes (1e-15 against
    4e-16) is recorded beside each figure: ~1e-12, because Brent from the same
    bracket stops at the same point of the band at any tight tolerance, so it
    does not measure which point of the band a second root finder stops at.
    Restarting from the reference's own post-regrid state brings one step back
    to L1 ~2e-11 (pressure)."""
    if not ref_available("jet2d"):
        pytest.skip("oracle/_ref/libref_jet2d.so not built")
    from oracle.refsim2d import run_isolated
    from gamma_b200 import gpu2d
    from helpers2d import energy
    p = dict(ncell=150, ntrack=5, nmax=300)
    with mp.get_context("spawn").Pool(1) as pool:
        d = pool.apply(_derived, (p,))
        before, after = pool.apply(_ref_after_regrid, (p,))
    th, dth = theta_of(before)
    g = gpu2d.Grid2DGPU(len(th), p["nmax"], th, dth)
    g.set_params(params_of(p, d))
    g.upload(state_from_reference(before))
    g.prepare()
    got = g.download()
    assert _same_counts(got, after)
    nmerged = sum(b.ntrack for b in before.tracks) - sum(a.ntrack for a in after.tracks)
    assert nmerged > 100
    for j in range(2, len(after.tracks) - 2):
        a, b = got.track(j), after.tracks[j]
        assert np.array_equal(a["x"], b.x) and np.array_equal(a["dx"], b.dx), j
        assert np.array_equal(a["xI"], b.xI), j
        E = energy(b.prim)
        assert np.all(np.abs(a["prim"][0] - b.prim[0]) <= 1e-13 * b.prim[0]), j
        assert np.all(np.abs(a["prim"][1] - b.prim[1]) <= np.maximum(1e-13 * b.prim[1], 1e-15 * E)), j
        for q in (4, 6, 7):
            assert np.all(np.abs(a["prim"][q] - b.prim[q]) <= 1e-13 * np.abs(b.prim[q])), (j, q)
    g.close()
    # then whole steps
    snaps = run_isolated(p, snap_at=(0, 1, 4), c2p_epsrel=EPS_CONVERGED)
    alt = run_isolated(p, snap_at=(0, 1, 4), c2p_epsrel=1e-15)
    g = gpu2d.Grid2DGPU(len(th), p["nmax"], th, dth)
    g.set_params(params_of(p, d))
    g.upload(state_from_reference(snaps[0]))
    for k in (1, 4):
        st = g.step(1 if k == 1 else 3)
        got = g.download()
        assert st["status"] == 0
        assert _same_counts(got, snaps[k])
        qs = (0, 1, 2, 4, 6, 7)
        bar = {q: 1e-6 if q in (6, 7) else 1e-7 for q in qs}
        l1 = l1_by_quantity(got, snaps[k], qs=qs)
        self_l1 = l1_between_snapshots(alt[k], snaps[k], qs)
        for q in qs:
            record(f"step {k} L1 slot {q} (reference tolerance sensitivity {self_l1[q]:.2e})", l1[q], bar[q])
        assert all(l1[q] <= bar[q] for q in qs), (k, l1, self_l1)
    g.close()
