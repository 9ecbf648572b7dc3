"""Golden fixtures written by the GAMMA reference itself (tests/golden/make_golden.py,
run where the reference sources are): the oracle restatement must reproduce
them bit for bit, and the GPU path within the parity bars.  These tests need
neither the reference sources nor its compiled build."""
import ast
import os

import numpy as np
import pytest

from helpers import l1_rel

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("prim", "x", "dx", "dt_loc", "sd", "shocked", "xI")


def _load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)
    params = ast.literal_eval(str(z["params"]))  # the dict written by make_golden.py
    return z, params


def _snap(z, k):
    t, dt, it, n = z[f"s{k}_scalars"]
    return dict(t=t, dt=dt, it=int(it), ntrack=int(n), **{f: z[f"s{k}_{f}"] for f in FIELDS})


@pytest.mark.parametrize("name,kind", [("tube", "tube"), ("bm1d", "bm1d")])
def test_oracle_restatement_reproduces_golden(name, kind):
    from oracle import port
    z, params = _load(name)
    cfg = port.tube_config(**params) if kind == "tube" else port.bm1d_config(**params)
    s = port.PortSim(cfg)
    s.init()
    done = 0
    for k in [int(v) for v in z["steps"]]:
        s.step(k - done)
        done = k
        got, want = s.snapshot(), _snap(z, k)
        assert got.ntrack == want["ntrack"] and got.t == want["t"] and got.dt == want["dt"], (name, k)
        for f in FIELDS:
            assert np.array_equal(getattr(got, f), want[f], equal_nan=True), (name, k, f)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tube", "bm1d"])
def test_gpu_reproduces_golden(gpu_available, name):
    from gamma_b200 import gpu, problems
    z, params = _load(name)
    if name == "tube":
        setup, cfg = problems.TubeSetup(**params), gpu.config_cart()
    else:
        setup, cfg = problems.Bm1dSetup(**params), gpu.config_sph()
    st0 = setup.initial_state()
    w0 = _snap(z, 0)
    assert st0.ntrack == w0["ntrack"] and np.array_equal(st0.x, w0["x"])
    g = gpu.GammaGPU(cfg, [setup.capacity])
    if name == "bm1d":
        g.set_params([setup.run_params()])
    pk = problems.pack([st0], g.offsets, g.total, cfg.nq)
    g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])
    done = 0
    for k in [int(v) for v in z["steps"]][1:]:
        assert g.step(k - done)["status"] == 0
        done = k
        got, want = problems.unpack(g.download(), 0, g.offsets), _snap(z, k)
        assert got.ntrack == want["ntrack"], (name, k)
        assert abs(got.t - want["t"]) <= 1e-13 * want["t"]
        a = slice(2, got.ntrack - 2)
        for q in (0, 1, 2):
            assert l1_rel(got.prim[q, a], want["prim"][q, a]) <= 1e-9, (name, k, q)
    g.close()


@pytest.mark.gpu
def test_gpu_2d_reproduces_golden(gpu_available):
    """The smoke check's 2D wedge against the reference's converged 2D step."""
    from gamma_b200 import gpu2d, problems
    z, params = _load("jet2d")
    p = dict(params)
    p["ntheta"] = p.pop("ntrack")
    s = problems.Jet2dSetup(**p)
    th, dth = s.theta()
    g = gpu2d.Grid2DGPU(s.ntheta, s.nmax, th, dth)
    g.set_params(s.params())
    g.upload(s.initial_state(), run_ghosts=True)
    k = int(z["steps"][-1])
    assert g.step(k)["status"] == 0
    got = g.download()
    g.close()
    for q in (0, 1):
        num = den = 0.
        for j in range(2, int(z[f"s{k}_ntracks"]) - 2):
            n = int(z[f"s{k}_j{j}_n"])
            assert int(got.ntrack[j]) == n, j
            ref = z[f"s{k}_j{j}_prim"][q, 2:n - 2]
            num += np.sum(np.abs(got.prim[q, j * got.cap + 2:j * got.cap + n - 2] - ref))
            den += np.sum(np.abs(ref))
        assert num / den < 1e-8, (q, num / den)
