"""Text snapshots against the reference's own IO module.

The oracle builds oracle/_ref/libref_{bm1d,tube,jet2d}_io.so link the
reference's src/IO/text1d.cpp / text2d.cpp.  There, Grid::printCols writes
../results/Last/phys%010d.out relative to the working directory (each reference
run works in its own temporary tree) and Simu::reinitialise reads the last dump
back.  The library's writer must produce the same bytes from the same state,
and its reader the same state the reference's resume builds.  Host code only:
no GPU is needed.
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

from conftest import ref_available

BM = dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, ncell=300, nmax=600, grid_log=1, r_lo=0.98, r_hi=1.02)
TUBE = dict(ncell=400, nmax=400, vL=0.3, vR=0.3, rhoL=10.0)
JET = dict(ncell=60, ntrack=6, nmax=120, split_DR=2.5, merge_DR=0.3, split_DR_slow=2.5, merge_DR_slow=0.3)


def _tree(root):
    os.makedirs(os.path.join(root, "results", "Last"), exist_ok=True)
    os.makedirs(os.path.join(root, "bin"), exist_ok=True)
    return os.path.join(root, "results", "Last")


def _ref_dump_1d(kind, params, steps, root):
    """A reference run that dumps at `steps` (printCols) in its own tree."""
    _tree(root)
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim import RefSim
    s = RefSim(kind)
    s.set_params(**params)
    s.init()
    s.step(steps)
    s.print_cols()
    return s.snapshot(), s.scalars()


def _ref_resume_1d(kind, params, root):
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim import RefSim
    s = RefSim(kind)
    s.set_params(**params)
    s.resume()
    return s.snapshot(), s.scalars()


def _ref_dump_2d(params, steps, root):
    _tree(root)
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim2d import RefJet2D
    s = RefJet2D(io=True)
    s.set_params(**params)
    s.init()
    s.step(steps)
    s.print_cols()
    return s.snapshot()


def _ref_resume_2d(params, root):
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim2d import RefJet2D
    s = RefJet2D(io=True)
    s.set_params(**params)
    s.resume()
    return s.snapshot()


def _in_ref_process(fn, *args):
    with mp.get_context("spawn").Pool(1) as pool:
        return pool.apply(fn, args)


@pytest.mark.parametrize("kind", ["bm1d_io", "tube_io"])
def test_text1d_dump_and_resume_match_reference(kind, tmp_path):
    if not ref_available(kind):
        pytest.skip(f"oracle/_ref/libref_{kind}.so not built")
    from gamma_b200 import gpu, problems
    steps = 7
    params = BM if kind == "bm1d_io" else TUBE
    snap, sc = _in_ref_process(_ref_dump_1d, kind, params, steps, str(tmp_path))
    it = int(sc["it"])
    ref_file = os.path.join(tmp_path, "results", "Last", f"phys{it:010d}.out")
    assert os.path.exists(ref_file)
    # writer: the reference's state after its printCols (slot TR1+1 holds what it stored)
    cfg = gpu.config_sph() if kind == "bm1d_io" else gpu.config_cart()
    mine = str(tmp_path / "mine.out")
    gpu.text1d_write(mine, cfg, snap.prim[:cfg.nq], snap.x, snap.dx, it, snap.t)
    want, got = open(ref_file, "rb").read(), open(mine, "rb").read()
    assert got.count(b"\n") == snap.ntrack - 4 + 1
    assert got == want
    # reader: the -r start of both from that file (read here first: the
    # reference's resume dumps again, over the same name)
    setup = problems.Bm1dSetup(**params) if kind == "bm1d_io" else problems.TubeSetup(**params)
    st = setup.resume_state(ref_file)
    ref_snap, ref_sc = _in_ref_process(_ref_resume_1d, kind, params, str(tmp_path))
    assert st.ntrack == ref_snap.ntrack and st.it == int(ref_sc["it"]) == it and st.t == ref_sc["t"]
    n = st.ntrack
    assert np.array_equal(st.x, ref_snap.x[:n]) and np.array_equal(st.dx, ref_snap.dx[:n])
    assert np.array_equal(st.xI, ref_snap.xI[:n - 1])
    for q in range(cfg.nq):
        assert np.array_equal(st.prim[q], ref_snap.prim[q, :n]), q


def test_text2d_dump_and_resume_match_reference(tmp_path):
    if not ref_available("jet2d_io"):
        pytest.skip("oracle/_ref/libref_jet2d_io.so not built")
    from gamma_b200 import gpu2d
    from helpers2d import state_from_reference, theta_of
    steps = 4
    snap = _in_ref_process(_ref_dump_2d, JET, steps, str(tmp_path))
    ref_file = os.path.join(tmp_path, "results", "Last", f"phys{snap.it:010d}.out")
    assert os.path.exists(ref_file)
    s = state_from_reference(snap)
    th, dth = theta_of(snap)
    mine = str(tmp_path / "mine2d.out")
    gpu2d.text2d_write(mine, s, th, dth)
    assert open(mine, "rb").read() == open(ref_file, "rb").read()
    # reader: active tracks and cells as the reference's resume leaves them
    # (read here first: the reference's resume dumps again, over the same name)
    got, gth, gdth = gpu2d.text2d_read(ref_file, len(th), JET["nmax"])
    ref = _in_ref_process(_ref_resume_2d, JET, str(tmp_path))
    assert got.it == ref.it and got.t == ref.t
    rth, rdth = theta_of(ref)  # the file's 16 digits, not the run's own theta
    assert np.array_equal(gth, rth) and np.array_equal(gdth, rdth)
    assert np.allclose(gth, th, rtol=1e-15, atol=0) and np.allclose(gdth, dth, rtol=1e-15, atol=0)
    for j in range(2, len(ref.tracks) - 2):
        t = ref.tracks[j]
        a = got.track(j)
        assert a["n"] == t.ntrack, j
        act = slice(2, t.ntrack - 2)
        assert np.array_equal(a["x"][act], t.x[act]) and np.array_equal(a["dx"][act], t.dx[act]), j
        assert np.array_equal(a["xI"][1:t.ntrack - 2], t.xI[1:t.ntrack - 2]), j
        for q in range(10):
            if q == 5:  # the resume's printCols stored Sd (-1, a new Cell's) there
                assert np.all(t.prim[q, act] == -1.) and np.all(a["prim"][q, act] == 0.), j
                continue
            assert np.array_equal(a["prim"][q, act], t.prim[q, act]), (j, q)


def test_text_reader_rejects_bad_files(tmp_path):
    from gamma_b200 import gpu
    bad = tmp_path / "phys0000000003.out"
    bad.write_text("t nact i x dx dlx rho vx p D sx tau trac Sd gmin gmax\n1 2 3\n")
    with pytest.raises(gpu.GammaError):
        gpu.text1d_read(str(bad), gpu.config_sph(), 100)
    with pytest.raises(gpu.GammaError):
        gpu.text1d_read(str(tmp_path / "missing.out"), gpu.config_sph(), 100)
    big = tmp_path / "phys0000000004.out"
    line = " ".join(["1.0", "500", "499"] + ["1.0"] * 13)
    big.write_text("header\n" + line + "\n")
    with pytest.raises(gpu.GammaError):  # more cells than the capacity
        gpu.text1d_read(str(big), gpu.config_sph(), 100)


def test_text1d_large_dump_matches_reference(tmp_path):
    """50,000 cells: the writer formats and the reader parses in several host
    threads; the bytes and the resumed state are still the reference's (its
    initial dump, iteration 0)."""
    if not ref_available("bm1d_io"):
        pytest.skip("oracle/_ref/libref_bm1d_io.so not built")
    from gamma_b200 import gpu
    params = dict(BM, ncell=50000, nmax=60000)
    snap, sc = _in_ref_process(_ref_dump_1d, "bm1d_io", params, 0, str(tmp_path))
    ref_file = os.path.join(tmp_path, "results", "Last", "phys0000000000.out")
    mine = str(tmp_path / "mine.out")
    gpu.text1d_write(mine, gpu.config_sph(), snap.prim, snap.x, snap.dx, 0, snap.t)
    assert open(mine, "rb").read() == open(ref_file, "rb").read()
    # the reader parses in several threads too
    from gamma_b200 import problems
    st = problems.Bm1dSetup(**params).resume_state(ref_file)
    ref_snap, _ = _in_ref_process(_ref_resume_1d, "bm1d_io", params, str(tmp_path))
    n = st.ntrack
    assert n == ref_snap.ntrack
    assert np.array_equal(st.prim, ref_snap.prim[:, :n]) and np.array_equal(st.xI, ref_snap.xI[:n - 1])
