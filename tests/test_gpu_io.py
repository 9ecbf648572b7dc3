"""Snapshots on the GPU path: the dump of a device run, the reference's resume
workflow end to end, and the exact binary checkpoints (1D runs and the 2D grid).
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

from conftest import ref_available
from helpers import l1_rel, record

pytestmark = pytest.mark.gpu

BM = dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, ncell=300, nmax=600, grid_log=1, r_lo=0.98, r_hi=1.02)


def _ref_dump_then_resume(params, k, m, root):
    """The reference (its own text IO linked): k steps, printCols; then, in a
    fresh Simu from that file (main.cpp -r), m more steps."""
    os.makedirs(os.path.join(root, "results", "Last"), exist_ok=True)
    os.makedirs(os.path.join(root, "bin"), exist_ok=True)
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim import RefSim
    s = RefSim("bm1d_io")
    s.set_params(**params)
    s.init()
    s.step(k)
    s.print_cols()
    it = int(s.scalars()["it"])
    path = os.path.join(root, "results", "Last", f"phys{it:010d}.out")
    with open(path, "rb") as f:
        dump = f.read()
    return s.snapshot(), dump


def _ref_resume_steps(params, m, root):
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim import RefSim
    s = RefSim("bm1d_io")
    s.set_params(**params)
    s.resume()
    s.step(m)
    return s.snapshot()


def _pool():
    return mp.get_context("spawn").Pool(1)


def _bm_context(setup):
    from gamma_b200 import gpu
    g = gpu.GammaGPU(gpu.config_sph(), [setup.capacity])
    g.set_params([setup.run_params()])
    return g


def _upload(g, states, nq):
    from gamma_b200 import problems
    pk = problems.pack(states, g.offsets, g.total, nq)
    g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])


def test_bm1d_resume_from_reference_dump(gpu_available, tmp_path):
    """main.cpp's -r workflow across implementations: the reference dumps at
    step 5; the GPU path resumes from that file and takes 15 steps; the
    reference resumes from the same file and takes the same steps."""
    if not ref_available("bm1d_io"):
        pytest.skip("oracle/_ref/libref_bm1d_io.so not built")
    from gamma_b200 import problems
    root = str(tmp_path)
    with _pool() as pool:
        _, dump = pool.apply(_ref_dump_then_resume, (BM, 5, 15, root))
    mine = tmp_path / "phys0000000005.out"
    mine.write_bytes(dump)
    setup = problems.Bm1dSetup(**BM)
    st = setup.resume_state(str(mine))
    with _pool() as pool:
        ref = pool.apply(_ref_resume_steps, (BM, 15, root))
    g = _bm_context(setup)
    _upload(g, [st], 10)
    stats = g.step(15)
    assert stats["status"] == 0
    got = problems.unpack(g.download(), 0, g.offsets)
    g.close()
    assert got.ntrack == ref.ntrack and got.it == ref.it
    # 15 time steps, each the CFL minimum over cold-gas wave speeds
    record("relative time difference after 15 steps", abs(got.t - ref.t) / ref.t, 1e-12)
    assert abs(got.t - ref.t) <= 1e-12 * ref.t
    a = slice(2, got.ntrack - 2)
    record("L1 max over slots", max(l1_rel(got.prim[q, a], ref.prim[q, a]) for q in (0, 1, 2, 4, 6, 7)), 1e-8)
    for q in (0, 1, 2, 4, 6, 7):
        assert l1_rel(got.prim[q, a], ref.prim[q, a]) <= 1e-8, q


def test_bm1d_print_cols_marks_and_writes(gpu_available, tmp_path):
    """gamma_gpu_print_cols: slot TR1+1 takes isShocked on the device, and the
    file holds the host writer's columns of the run's state."""
    from gamma_b200 import gpu, problems
    setup = problems.Bm1dSetup(**BM)
    g = _bm_context(setup)
    _upload(g, [setup.initial_state()], 10)
    g.step(12)
    path = g.print_cols(0, str(tmp_path))
    assert os.path.basename(path) == "phys0000000012.out"
    out = problems.unpack(g.download(), 0, g.offsets)
    g.close()
    rows = np.loadtxt(path, skiprows=1, ndmin=2)
    assert rows.shape == (out.ntrack - 4, 16)
    sd = rows[:, 13]
    assert set(np.unique(sd)) <= {0., 1.} and sd.sum() > 0  # the blast wave's shock is marked
    assert np.array_equal(out.prim[5, 2:out.ntrack - 2], sd)
    mine = str(tmp_path / "host.out")
    gpu.text1d_write(mine, gpu.config_sph(), out.prim, out.x, out.dx, 12, out.t)
    assert open(mine, "rb").read() == open(path, "rb").read()


def test_checkpoint_continues_bit_exact(gpu_available, tmp_path):
    """save after 8 steps, 10 more steps; a fresh context loading the file and
    taking the same 10 steps lands on the same bits (two runs of uneven size)."""
    from gamma_b200 import gpu, problems
    setups = [problems.Bm1dSetup(**BM), problems.Bm1dSetup(**dict(BM, ncell=420, nmax=900, Etot=3e52))]
    caps = [s.capacity for s in setups]

    def ctx():
        g = gpu.GammaGPU(gpu.config_sph(), caps)
        g.set_params([s.run_params() for s in setups])
        return g
    g = ctx()
    _upload(g, [s.initial_state() for s in setups], 10)
    g.step(8)
    ck = str(tmp_path / "run.ckpt")
    g.save(ck)
    g.step(10)
    a = g.download()
    g.close()
    h = ctx()
    h.load(ck)
    h.step(10)
    b = h.download()
    h.close()
    assert np.array_equal(a["ntrack"], b["ntrack"]) and np.array_equal(a["it"], b["it"])
    assert np.array_equal(a["t"], b["t"])
    for r, (o, n) in enumerate(zip(g.offsets, a["ntrack"])):
        for k in ("x", "dx", "dt_loc"):
            assert np.array_equal(a[k][o:o + n], b[k][o:o + n]), (r, k)
        assert np.array_equal(a["xI"][o:o + n - 1], b["xI"][o:o + n - 1])
        assert np.array_equal(a["prim"][:, o:o + n], b["prim"][:, o:o + n]), r
    # a checkpoint of another layout is refused
    other = gpu.GammaGPU(gpu.config_sph(), [caps[0]])
    with pytest.raises(gpu.GammaError):
        other.load(ck)
    other.close()


def test_2d_checkpoint_and_dump(gpu_available, tmp_path):
    """2D: the checkpoint carries the gradients and the ghost cells' stale
    neighbour lists, so a loaded grid continues bit for bit; the dump marks Sd
    into slot TR1+1 and reads back through the reference-compatible reader."""
    from gamma_b200 import gpu2d, problems
    s = problems.Jet2dSetup(ncell=80, ntheta=6, nmax=160, split_DR=2.5, merge_DR=0.3, split_DR_slow=2.5,
                            merge_DR_slow=0.3)
    th, dth = s.theta()

    def ctx():
        g = gpu2d.Grid2DGPU(s.ntheta, s.nmax, th, dth)
        g.set_params(s.params())
        return g
    g = ctx()
    g.upload(s.initial_state(), run_ghosts=True)
    g.step(6)
    ck = str(tmp_path / "grid.ckpt")
    g.save(ck)
    g.step(7)
    a = g.download()
    h = ctx()
    h.load(ck)
    h.step(7)
    b = h.download()
    h.close()
    assert np.array_equal(a.ntrack, b.ntrack) and a.it == b.it and a.t == b.t
    for j in range(a.NJ):
        o, n = j * a.cap, int(a.ntrack[j])
        assert np.array_equal(a.prim[:, o:o + n], b.prim[:, o:o + n]), j
        assert np.array_equal(a.x[o:o + n], b.x[o:o + n]) and np.array_equal(a.xI[o:o + n - 1], b.xI[o:o + n - 1])
    # the dump
    path = g.print_cols(str(tmp_path))
    d = g.download()
    g.close()
    assert os.path.basename(path) == f"phys{d.it:010d}.out"
    for j in range(d.NJ):
        o, n = j * d.cap, int(d.ntrack[j])
        assert np.array_equal(d.prim[5, o:o + n], d.extra["sd"][o:o + n]), j
    back, bth, bdth = gpu2d.text2d_read(path, s.ntheta, s.nmax)
    assert np.array_equal(back.ntrack[2:-2], d.ntrack[2:-2])
    assert np.allclose(bth, th, rtol=1e-15, atol=0)
    for j in range(2, d.NJ - 2):
        o, n = j * d.cap, int(d.ntrack[j])
        act = slice(o + 2, o + n - 2)
        assert np.allclose(back.x[act], d.x[act], rtol=1e-15, atol=0)  # 16 significant digits
        assert np.allclose(back.prim[0, act], d.prim[0, act], rtol=1e-6)  # 7 digits


JET = dict(ncell=60, ntrack=6, nmax=120, split_DR=2.5, merge_DR=0.3, split_DR_slow=2.5, merge_DR_slow=0.3)


def _ref2d_dump(params, k, root):
    os.makedirs(os.path.join(root, "results", "Last"), exist_ok=True)
    os.makedirs(os.path.join(root, "bin"), exist_ok=True)
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim2d import RefJet2D
    s = RefJet2D(io=True)
    s.set_params(**params)
    s.init()
    s.step(k)
    s.print_cols()
    return s.derived()


def _ref2d_resume_steps(params, m, root):
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim2d import RefJet2D
    s = RefJet2D(io=True)
    s.set_params(**params)
    s.resume()
    s.set_c2p_epsrel(4e-16)
    s.step(m)
    return s.snapshot()


def test_2d_resume_from_reference_dump(gpu_available, tmp_path):
    """The 2D -r workflow across implementations: the reference dumps at step
    4 (7 significant digits for most columns); both resume from that file --
    default gradients and empty neighbour lists, ghosts from the ghost pass --
    and take 6 steps."""
    if not ref_available("jet2d_io"):
        pytest.skip("oracle/_ref/libref_jet2d_io.so not built")
    from gamma_b200 import gpu2d
    from helpers2d import l1_by_quantity, params_of
    root = str(tmp_path)
    with _pool() as pool:
        d = pool.apply(_ref2d_dump, (JET, 4, root))
    src = os.path.join(root, "results", "Last", "phys0000000004.out")
    st, th, dth = gpu2d.text2d_read(src, JET["ntrack"], JET["nmax"])
    with _pool() as pool:
        ref = pool.apply(_ref2d_resume_steps, (JET, 6, root))
    g = gpu2d.Grid2DGPU(JET["ntrack"], JET["nmax"], th, dth)
    g.set_params(params_of(JET, d))
    g.upload(st, run_ghosts=True)
    stats = g.step(6)
    got = g.download()
    g.close()
    assert stats["status"] == 0
    assert [int(got.ntrack[j]) for j in range(len(ref.tracks))] == [t.ntrack for t in ref.tracks]
    assert got.it == ref.it and abs(got.t - ref.t) <= 1e-13 * ref.t
    l1 = l1_by_quantity(got, ref, qs=(0, 1, 2, 4, 6, 7))
    assert all(v <= 1e-8 for v in l1.values()), l1
