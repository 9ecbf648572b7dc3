"""gamma_gpu_step_tubes_noalloc: the tube step for callers that cannot allocate.

A caller embedded in a framework that owns all device memory (or that must
not let cudaMalloc synchronise the device) passes its own device arrays; the
entry point keeps its workspace in a fixed device array inside the library.
Two calls in a row must give what the context-based entry point
(gamma_gpu_upload + gamma_gpu_step) gives for the same runs and steps.  The
same kernel runs on the same inputs in both cases -- only the order in which
CTAs pick runs differs, and runs are independent -- so the results are
required to be identical, not merely within the parity tolerance.

Collected last on purpose: if it fails, a run stopping at the first failure has
already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RUN_DTYPE = np.dtype([("ntrack", "<i4"), ("status", "<i4"), ("t", "<f8"), ("dt", "<f8"), ("it", "<i8")])
STORED_SLOTS = (0, 1, 2, 4, 5)  # slot 3 is not stored


def _setups():
    from gamma_b200 import problems
    return [problems.TubeSetup(ncell=n, vL=v, vR=v, rhoL=r) for n, v, r in
            ((64, 0.0, 10.0), (300, 0.3, 9.0), (1000, -0.4, 11.0), (2047, 0.1, 10.5), (129, 0.45, 8.2))]


def test_noalloc_step_matches_context_step(gpu_available):
    import torch

    from gamma_b200 import gpu, problems

    setups = _setups()
    states = [s.initial_state() for s in setups]
    cfg = gpu.config_cart()

    # reference: the context-based entry point
    g = gpu.GammaGPU(cfg, [s.capacity for s in setups])
    pk = problems.pack(states, g.offsets, g.total, 6)
    g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])
    expected = []
    for _ in range(2):
        st = g.step(2)
        assert st["status"] == 0
        expected.append((g.download(), st))
    offsets, total = g.offsets.copy(), g.total
    g.close()

    # the same runs in caller-owned device memory (the test allocates; the entry point does not)
    dev = torch.device("cuda", 0)
    d_prim = torch.tensor(np.ascontiguousarray(pk["prim"][list(STORED_SLOTS)]), device=dev)
    d_x = torch.tensor(pk["x"], device=dev)
    d_dx = torch.tensor(pk["dx"], device=dev)
    d_dtl = torch.tensor(pk["dt_loc"], device=dev)
    d_xI = torch.tensor(pk["xI"], device=dev)
    d_off = torch.tensor(offsets, dtype=torch.int64, device=dev)
    d_cap = torch.tensor([s.capacity for s in setups], dtype=torch.int32, device=dev)
    runs = np.zeros(len(setups), dtype=RUN_DTYPE)
    runs["ntrack"] = pk["ntrack"]
    runs["t"] = pk["t"]
    runs["it"] = pk["it"]
    d_runs = torch.tensor(np.frombuffer(runs.tobytes(), dtype=np.uint8), device=dev)
    ptrs = [d_off.data_ptr(), d_cap.data_ptr(), d_runs.data_ptr(), d_prim.data_ptr(), d_x.data_ptr(),
            d_dx.data_ptr(), d_dtl.data_ptr(), d_xI.data_ptr()]

    for call in range(2):
        st = gpu.step_tubes_noalloc(cfg, len(setups), total, *ptrs, nsteps=2)
        torch.cuda.synchronize()
        want, want_st = expected[call]
        assert st["status"] == 0
        assert st["zone_updates"] == want_st["zone_updates"]
        got_runs = np.frombuffer(d_runs.cpu().numpy().tobytes(), dtype=RUN_DTYPE)
        assert np.array_equal(got_runs["ntrack"], want["ntrack"])
        assert np.array_equal(got_runs["it"], want["it"])
        assert np.array_equal(got_runs["t"], want["t"])
        prim = d_prim.cpu().numpy()
        for r, s in enumerate(states):
            o, n = int(offsets[r]), int(want["ntrack"][r])
            for row, q in enumerate(STORED_SLOTS):
                assert np.array_equal(prim[row, o:o + n], want["prim"][q, o:o + n]), (call, r, q)
            for name, arr in (("x", d_x), ("dx", d_dx), ("dt_loc", d_dtl)):
                assert np.array_equal(arr.cpu().numpy()[o:o + n], want[name][o:o + n]), (call, r, name)
            assert np.array_equal(d_xI.cpu().numpy()[o:o + n - 1], want["xI"][o:o + n - 1]), (call, r)


def test_noalloc_rejects_batches_beyond_its_workspace(gpu_available):
    import torch

    from gamma_b200 import gpu

    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = d.data_ptr()
    with pytest.raises(gpu.GammaError) as e:
        gpu.step_tubes_noalloc(gpu.config_cart(), 1, 10_000_000, p, p, p, p, p, p, p, p, nsteps=1)
    assert e.value.code == gpu.GAMMA_ERR_CAPACITY
    # sizes whose workspace byte count would wrap a 64-bit size are rejected too
    with pytest.raises(gpu.GammaError) as e:
        gpu.step_tubes_noalloc(gpu.config_cart(), 1, 2 ** 62, p, p, p, p, p, p, p, p, nsteps=1)
    assert e.value.code == gpu.GAMMA_ERR_CAPACITY


def _device_runs(setups, states, offsets, total, dev):
    """Caller-owned device copies of packed tube runs (the test allocates them)."""
    import torch

    from gamma_b200 import problems

    pk = problems.pack(states, offsets, total, 6)
    arrs = dict(
        prim=torch.tensor(np.ascontiguousarray(pk["prim"][list(STORED_SLOTS)]), device=dev),
        x=torch.tensor(pk["x"], device=dev), dx=torch.tensor(pk["dx"], device=dev),
        dtl=torch.tensor(pk["dt_loc"], device=dev), xI=torch.tensor(pk["xI"], device=dev),
        off=torch.tensor(offsets, dtype=torch.int64, device=dev),
        cap=torch.tensor([s.capacity for s in setups], dtype=torch.int32, device=dev))
    runs = np.zeros(len(setups), dtype=RUN_DTYPE)
    runs["ntrack"] = pk["ntrack"]
    arrs["runs"] = torch.tensor(np.frombuffer(runs.tobytes(), dtype=np.uint8), device=dev)
    ptrs = [arrs[k].data_ptr() for k in ("off", "cap", "runs", "prim", "x", "dx", "dtl", "xI")]
    return arrs, ptrs


def _layout(setups):
    offsets, total = [], 0
    for s in setups:
        offsets.append(total)
        total += (s.capacity + 1) & ~1
    return np.array(offsets, dtype=np.int64), total


def test_noalloc_reports_negative_cfl_candidate(gpu_available):
    """A cell of negative width (the reference exits with code 30 there,
    cell.cpp:70-73): the call's stats say GAMMA_ERR_NEG_DT, the run's record
    keeps the reference code 30 and stops, the other run carries on -- with
    host stats and without them."""
    import torch

    from gamma_b200 import gpu, problems

    dev = torch.device("cuda", 0)
    setups = [problems.TubeSetup(ncell=64), problems.TubeSetup(ncell=80)]
    offsets, total = _layout(setups)
    for with_stats in (True, False):
        states = [s.initial_state() for s in setups]
        states[0].dx[10] = -abs(states[0].dx[10])
        arrs, ptrs = _device_runs(setups, states, offsets, total, dev)
        st = gpu.step_tubes_noalloc(gpu.config_cart(), len(setups), total, *ptrs, nsteps=3, stats=with_stats)
        torch.cuda.synchronize()
        if with_stats:
            assert st["status"] == gpu.GAMMA_ERR_NEG_DT
        else:
            assert st is None
        runs = np.frombuffer(arrs["runs"].cpu().numpy().tobytes(), dtype=RUN_DTYPE)
        assert runs["status"][0] == 30 and runs["status"][1] == 0
        assert runs["it"][0] == 1 and runs["it"][1] == 3


def test_context_steps_after_noalloc_call(gpu_available):
    """A context whose longest track needs more than 48 KB of dynamic shared
    memory (a 60,000-cell tube: the regrid bit words grow with the track)
    launches the same kernel as the no-alloc entry point.  A no-alloc call in
    between must leave the context able to step, and its results unchanged."""
    import torch

    from gamma_b200 import gpu, problems

    dev = torch.device("cuda", 0)
    big = [problems.TubeSetup(ncell=60_000, vL=0.2, vR=0.2)]
    states = [s.initial_state() for s in big]

    def run_context(noalloc_between):
        g = gpu.GammaGPU(gpu.config_cart(), [s.capacity for s in big])
        pk = problems.pack(states, g.offsets, g.total, 6)
        g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])
        assert g.step(1)["status"] == 0
        if noalloc_between:
            small = [problems.TubeSetup(ncell=64), problems.TubeSetup(ncell=100, vL=0.1, vR=0.1)]
            off, tot = _layout(small)
            arrs, ptrs = _device_runs(small, [s.initial_state() for s in small], off, tot, dev)
            assert gpu.step_tubes_noalloc(gpu.config_cart(), len(small), tot, *ptrs, nsteps=2)["status"] == 0
            torch.cuda.synchronize()
        st = g.step(2)
        out = g.download()
        g.close()
        return st, out

    want_st, want = run_context(False)
    got_st, got = run_context(True)
    assert got_st["status"] == 0 and got_st["zone_updates"] == want_st["zone_updates"]
    n = int(want["ntrack"][0])
    assert int(got["ntrack"][0]) == n
    assert np.array_equal(got["prim"][:, :n], want["prim"][:, :n])
    assert np.array_equal(got["xI"][:n - 1], want["xI"][:n - 1])
