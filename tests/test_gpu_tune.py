"""Launch shapes of the 1D step kernel and their autotuner
(gamma_gpu_set_variant, gamma_gpu_autotune).  Every shape computes every cell
the same way, so runs must agree bit for bit whatever the shape; the tuner must
leave the state it times as it found it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setups(kind):
    from gamma_b200 import problems
    if kind == "sph":
        base = dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, grid_log=1, r_lo=0.98, r_hi=1.02)
        return [problems.Bm1dSetup(**dict(base, ncell=n, nmax=2 * n, Etot=E)) for n, E in
                ((300, 1e53), (777, 3e52), (1500, 2e53))]
    return [problems.TubeSetup(ncell=n, vL=v, vR=v, rhoL=r) for n, v, r in
            ((300, 0.1, 10.0), (777, -0.3, 9.5), (1500, 0.45, 10.5))]


def _context(kind, setups):
    from gamma_b200 import gpu, problems
    cfg = gpu.config_sph() if kind == "sph" else gpu.config_cart()
    g = gpu.GammaGPU(cfg, [s.capacity for s in setups])
    if kind == "sph":
        g.set_params([s.run_params() for s in setups])
    pk = problems.pack([s.initial_state() for s in setups], g.offsets, g.total, cfg.nq)
    g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])
    return g


def _same(a, b, offsets):
    assert np.array_equal(a["ntrack"], b["ntrack"]) and np.array_equal(a["t"], b["t"])
    for o, n in zip(offsets, a["ntrack"]):
        assert np.array_equal(a["prim"][:, o:o + n], b["prim"][:, o:o + n])
        assert np.array_equal(a["x"][o:o + n], b["x"][o:o + n])
        assert np.array_equal(a["xI"][o:o + n - 1], b["xI"][o:o + n - 1])
        assert np.array_equal(a["dt_loc"][o:o + n], b["dt_loc"][o:o + n])


@pytest.mark.parametrize("kind", ["sph", "cart"])
def test_every_launch_shape_gives_the_same_bits(gpu_available, kind):
    from gamma_b200 import gpu
    setups = _setups(kind)
    outs = []
    for v in range(gpu.N_VARIANTS):
        g = _context(kind, setups)
        g.set_variant(v)
        st = g.step(20)
        assert st["status"] == 0 and g.variant == v
        outs.append((g.download(), st))
        offsets = g.offsets
        g.close()
    for v in range(1, gpu.N_VARIANTS):
        _same(outs[0][0], outs[v][0], offsets)
        assert outs[v][1]["zone_updates"] == outs[0][1]["zone_updates"], v


def test_autotune_restores_the_state_and_keeps_the_fastest(gpu_available):
    from gamma_b200 import gpu
    setups = _setups("sph")
    g = _context("sph", setups)
    g.step(3)
    before = g.download()
    ms, chosen = g.autotune(4)
    assert len(ms) == gpu.N_VARIANTS and all(t > 0 for t in ms)
    assert g.variant == chosen and ms[chosen] <= ms[0]
    assert chosen == 0 or ms[chosen] < 0.97 * ms[0]
    _same(before, g.download(), g.offsets)  # the state it timed is put back
    g.step(10)
    a = g.download()
    offsets = g.offsets
    g.close()
    h = _context("sph", setups)
    h.step(13)
    _same(a, h.download(), offsets)
    h.close()


def test_graph_replay_gives_the_same_bits(gpu_available):
    """Step calls replayed from the captured graph (the default), recaptured
    when the step count or the shape changes, against direct launches."""
    setups = _setups("sph")
    outs = []
    for graphs in (True, False):
        g = _context("sph", setups)
        g.use_graphs(graphs)
        for k, v in ((3, 0), (1, 0), (1, 0), (4, 2), (2, 0)):
            g.set_variant(v)
            assert g.step(k)["status"] == 0
        outs.append(g.download())
        offsets = g.offsets
        g.close()
    _same(outs[0], outs[1], offsets)
