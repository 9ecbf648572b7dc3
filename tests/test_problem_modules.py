"""Problem modules (include/gamma_problem.h): the registry and the host-side
set-up hooks, against the reference's own initialisation.  No GPU needed:
gamma_gpu_problem_id and gamma_gpu_initial_state run on the host.

isen1d is the reference's Tests/isen1D.cpp as a module of the library;
hooked_tube is a module compiled from outside the library's sources
(tests/modules/hooked_tube.cu, built into gamma_b200/lib/libgamma_b200_hooked.so
with make INITIAL=...), mirrored by oracle/ref_harness/hooked_tube_cfg.cpp."""
import ctypes
import multiprocessing as mp
import os

import numpy as np
import pytest

from conftest import ROOT, ref_available

HOOKED_LIB = os.path.join(ROOT, "gamma_b200", "lib", "libgamma_b200_hooked.so")
# hooked_tube parameter words, in the order of tests/modules/hooked_tube.cu
HOOKED = dict(g=0.5, p_floor=2.e-3, v_out=0.2, split_dx=1.6e-3, merge_dx=0.6e-3, ncell=1000., nmax=2000., xmin=0.1,
              xmax=1.1, xmid=0.6, rhoL=10., pL=13.33, vL=0.3, rhoR=1., pR=1.e-3, vR=0., reflect=1., wall=1.)


def hooked_words(p=HOOKED):
    return [float(p[k]) for k in ("g", "p_floor", "v_out", "split_dx", "merge_dx", "ncell", "nmax", "xmin", "xmax",
                                  "xmid", "rhoL", "pL", "vL", "rhoR", "pR", "vR", "reflect", "wall")]


def _ref_initial(kind, params):
    from oracle.refsim import RefSim
    s = RefSim(kind)
    s.set_params(**params)
    s.init()
    return s.snapshot()


def ref_initial(kind, params):
    with mp.get_context("spawn").Pool(1) as pool:
        return pool.apply(_ref_initial, (kind, params))


def _same_as_reference(got, snap):
    nt, t, prim, x, dx, xI, dtl = got
    assert nt == snap.ntrack and t == snap.t
    assert np.array_equal(prim[:, :nt], snap.prim)
    assert np.array_equal(x[:nt], snap.x) and np.array_equal(dx[:nt], snap.dx)
    assert np.array_equal(xI[:nt - 1], snap.xI)
    assert np.all(dtl[:nt] == 1e15)


def test_registry_names_the_modules():
    from gamma_b200 import gpu
    assert gpu.problem_id("bm1d") == gpu.PROBLEM_BM1D
    assert gpu.problem_id("tube") == gpu.PROBLEM_TUBE
    assert gpu.problem_id("isen1d") >= 16
    with pytest.raises(KeyError):
        gpu.problem_id("no_such_problem")
    # a module runs only with the module set it was built for
    with pytest.raises(gpu.GammaError) as e:
        gpu.initial_state(gpu.config_sph(), [0.] * 10, 4000)  # bm1d: set up in Python, not by hooks
    assert e.value.code == gpu.GAMMA_ERR_INVALID
    cfg = gpu.config_sph()
    cfg.problem = gpu.problem_id("isen1d")  # a cartesian module
    with pytest.raises(gpu.GammaError):
        gpu.initial_state(cfg, [0.] * 10, 4000)


def test_isen1d_initial_state_is_the_reference_one():
    """isen1D.cpp's loadParams, initialGeometry and initialValues (with the
    reference's own constants: zero parameter words), then prepForRun and the
    first updateGhosts, bit for bit."""
    if not ref_available("isen1d"):
        pytest.skip("oracle/_ref/libref_isen1d.so not built")
    from gamma_b200 import gpu
    cfg = gpu.config_cart(problem=gpu.problem_id("isen1d"))
    got = gpu.initial_state(cfg, [0.] * 10, 3160 + 50 + 4)
    _same_as_reference(got, ref_initial("isen1d", {}))
    with pytest.raises(gpu.GammaError) as e:  # capacity below nmax + 2 ngst
        gpu.initial_state(cfg, [0.] * 10, 3000)
    assert e.value.code == gpu.GAMMA_ERR_CAPACITY


def test_module_from_outside_the_library_sources():
    """The INITIAL-built library holds the built-in modules and hooked_tube;
    hooked_tube's set-up equals the reference harness's bit for bit."""
    if not os.path.exists(HOOKED_LIB):
        pytest.skip("libgamma_b200_hooked.so not built")
    from gamma_b200 import gpu
    L = ctypes.CDLL(HOOKED_LIB)
    L.gamma_gpu_problem_id.argtypes = [ctypes.c_char_p]
    ids = {n: L.gamma_gpu_problem_id(n.encode()) for n in ("bm1d", "tube", "isen1d", "hooked_tube")}
    assert ids["bm1d"] == 0 and ids["tube"] == 1 and ids["isen1d"] >= 16 and ids["hooked_tube"] >= 16
    assert ids["isen1d"] != ids["hooked_tube"]
    if not ref_available("hooked_tube"):
        pytest.skip("oracle/_ref/libref_hooked_tube.so not built")
    cfg = gpu.config_cart(problem=ids["hooked_tube"])
    cap = int(HOOKED["nmax"]) + 4
    w = np.ascontiguousarray(hooked_words(), dtype=np.float64)
    prim = np.zeros((6, cap))
    x, dx, xI, dtl = (np.zeros(cap) for _ in range(4))
    nt, t = ctypes.c_int(), ctypes.c_double()
    dp = ctypes.POINTER(ctypes.c_double)
    L.gamma_gpu_initial_state.argtypes = [ctypes.POINTER(gpu.Config), dp, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int), dp, dp, dp, dp, dp, dp]
    rc = L.gamma_gpu_initial_state(ctypes.byref(cfg), w.ctypes.data_as(dp), w.size, cap, ctypes.byref(nt),
                                   ctypes.byref(t), *(a.ctypes.data_as(dp) for a in (prim, x, dx, xI, dtl)))
    assert rc == 0
    _same_as_reference((nt.value, t.value, prim, x, dx, xI, dtl), ref_initial("hooked_tube", HOOKED))


def test_shim_compiles_against_the_reference_headers():
    """gamma_b200/shim/simu_b200.cpp (the reference's Simu with its loop on the
    device) compiles against the reference's own headers and links with the
    reference's sources, Tests/BM1D.cpp and libgamma_b200.so."""
    import subprocess
    ref = os.environ.get("GAMMA_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
    if not os.path.isdir(os.path.join(ref, "src")):
        pytest.skip("reference sources not present")
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "_ref/shim_bm1d", f"REF={ref}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert os.access(os.path.join(ROOT, "oracle", "_ref", "shim_bm1d"), os.X_OK)
