"""Benchmark: zone-updates/s of the moving-mesh relativistic hydro step on B200.

Workload (one GPU): 4096 independent planar relativistic shock tubes
(cartesian + rel_cart, Gamma = 5/3, NUM_Q = 6, no regrid), each with a seeded
cell count drawn log-uniformly from 256-8192, rho_L = 10 and p_L = 13.33 with
+-20 % jitter, rho_R = 1, p_R = 1e-7 and one initial velocity U(-0.5, 0.5)
applied to both states.  A step is one RK3 step of every tube, each with its own
dt, in one persistent launch.  Synthetic inputs stand in for the reference's
problem setups; the state (~1.4 GB) is larger than L2, so every step streams it
from HBM.

Arms:
  (default)          the CUDA path: `value` times steps on device-resident state;
                     `e2e` times the C-ABI job from pinned host buffers (upload,
                     steps, download).
  --impl reference   the reference's own CPU implementation of the step
                     (oracle/_ref, compiled from the reference sources; the C
                     restatement if that build is absent) on a bounded sample of
                     tubes, one process per host core.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NTUBES = 4096
SEED = 20241203
B_ZU_NQ6 = 8 * (8 * (6 + 1) + 1)  # algorithmic bytes per zone-update (456 for NUM_Q = 6)
B_ZU_NQ10 = 8 * (8 * (10 + 1) + 1)  # 712 for NUM_Q = 10
METRIC = "zone-updates/s on 1 B200: plain vs batched+learned c2p at L1<=1e-8; HBM % peak"


def tube_setups(ntubes=NTUBES, seed=SEED):
    from gamma_b200 import problems
    rng = np.random.default_rng(seed)
    n = np.floor(np.exp(rng.uniform(math.log(256), math.log(8192), ntubes))).astype(int)
    jr = rng.uniform(-0.2, 0.2, ntubes)
    jp = rng.uniform(-0.2, 0.2, ntubes)
    v = rng.uniform(-0.5, 0.5, ntubes)
    return [problems.TubeSetup(ncell=int(n[i]), rhoL=10. * (1. + jr[i]), pL=13.33 * (1. + jp[i]), vL=float(v[i]),
                               vR=float(v[i]), rhoR=1.0, pR=1.e-7) for i in range(ntubes)]


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi SM clock / throttle-reason samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.n_before = 0

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.perf_counter()  # the first sample marks the start of the timed region
            while not self.rows and self.proc.poll() is None and time.perf_counter() - t0 < 5.:
                time.sleep(0.01)
            self.n_before = len(self.rows)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            # a region shorter than the sampling period still gets the sample that follows it
            t0 = time.perf_counter()
            while len(self.rows) <= self.n_before and self.proc.poll() is None and time.perf_counter() - t0 < 1.:
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in self.rows for j in range(4) if r[3 + j].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_zone():
    """DRAM bytes per zone-update of the step kernel from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return float(json.load(f)["track_step_cart_dram_bytes_per_zone_update"])
    except (OSError, KeyError, ValueError):
        return None


# ---------------------------------------------------------------------------
# CPU arms (the reference's own code, or the restatement)

def _cpu_worker(args):
    kind, tubes, steps, warmup = args
    sys.path.insert(0, ROOT)
    zones = 0
    t_total = 0.0
    for t in tubes:
        if kind == "reference":  # one process-wide Simu per library: re-initialised per tube
            from oracle.refsim import RefSim
            s = RefSim("tube")
            s.set_params(**t)
            s.init()
        else:
            from oracle import port
            s = port.PortSim(port.tube_config(**t))
            s.init()
        s.step(warmup)
        t0 = time.perf_counter()
        s.step(steps)
        t_total += time.perf_counter() - t0
        zones += steps * int(t["ncell"])
    return zones, t_total


def cpu_run(setups, steps, warmup, sample, cores, budget_zones):
    """Time the CPU step on a sample of tubes, one process per core; returns (zone-updates/s, info)."""
    import multiprocessing as mp

    kind = "reference" if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_tube.so")) else "port"
    rng = np.random.default_rng(SEED + 1)
    idx = rng.choice(len(setups), size=min(sample, len(setups)), replace=False)
    tubes = []
    for i in idx:
        s = setups[i]
        tubes.append(dict(ncell=s.ncell, nmax=s.ncell, rhoL=s.rhoL, pL=s.pL, vL=s.vL, vR=s.vR, rhoR=s.rhoR, pR=s.pR))
    # bound the work: scale the step count so the sample is ~budget_zones zone-updates
    zsum = sum(t["ncell"] for t in tubes)
    steps = max(1, min(steps, int(budget_zones // max(zsum, 1))))
    chunks = [tubes[k::cores] for k in range(cores)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(kind, ch, steps, warmup) for ch in chunks if ch])
    wall = time.perf_counter() - t0
    zones = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    value = zones / busy
    info = {"kind": kind, "cores": cores,
            "sample": f"{len(tubes)} of the {len(setups)} tubes (seeded), {steps} timed RK3 steps each after "
                      f"{warmup} warm-up steps, {cores} processes; value = sample zone-updates / slowest process"}
    return value, info, wall


# ---------------------------------------------------------------------------

def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    setups = tube_setups()
    cores = os.cpu_count() or 1
    steps = max(1, args.steps)
    value, info, wall = cpu_run(setups, steps, args.warmup, sample=max(64, cores * 2), cores=cores,
                                budget_zones=float(os.environ.get("GAMMA_REF_ZONES", 4.0e7)))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "4096 cartesian relativistic shock tubes, 256-8192 cells (log-uniform), "
                                   "Gamma=5/3, NUM_Q=6, one RK3 step per step", "tubes": NTUBES, "seed": SEED},
            "cpu_baseline": dict(info, value=value, unit="zone-updates/s"),
            "e2e": {"value": value, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# kernel launches of one 2D step (gamma_2d.cu enqueue_step_until): 4 regrid,
# 16 per RK3 stage, collect_dt's 2 in stage 1, the advance
LAUNCHES_2D = 4 + 3 * 16 + 2 + 1
JET2D = dict(ntheta=512, ncell=12000, nmax=12000)  # tracks settle at ~3,000-4,000 cells after the first regrid
# the sweep workload's large 2D case: slow cells merge only below 0.3 of the
# target spacing, so the tracks keep ~8,000 cells (~33 M zones)
JET2D_C4 = dict(ntheta=4096, ncell=8000, nmax=8400, merge_DR_slow=0.3)


def _jet2d_cpu_worker(args):
    """The reference's own 2D step (oracle/_ref/libref_jet2d.so) on a narrower wedge."""
    params, steps, warmup = args
    sys.path.insert(0, ROOT)
    from oracle.refsim2d import RefJet2D
    s = RefJet2D()
    s.set_params(**params)
    s.init()
    s.step(warmup)
    n0 = sum(t.ntrack - 4 for t in s.snapshot().tracks[2:-2])
    t0 = time.perf_counter()
    s.step(steps)
    dt = time.perf_counter() - t0
    n1 = sum(t.ntrack - 4 for t in s.snapshot().tracks[2:-2])
    return steps * 0.5 * (n0 + n1), dt


def _jet2d_run(s, steps, warmup, guess_ptr=0, dev_index=None, after=None, graphs=True):
    """Fresh 2D grid from the initial state: warm-up steps, one step with
    statistics, then `steps` timed steps (statistics over them), each one graph
    launch (graphs) or its kernels launched one by one; after(grid) runs
    before the grid is released."""
    import torch

    from gamma_b200 import gpu2d
    th, dth = s.theta()
    g = gpu2d.Grid2DGPU(s.ntheta, s.nmax, th, dth)
    g.set_params(s.params())
    g.set_guess(guess_ptr)
    g.use_graphs(graphs)
    g.upload(s.initial_state(), run_ghosts=True)
    for _ in range(max(warmup, 3)):
        g.step(1, stats=False)
    st0 = g.step(1)
    assert st0["status"] == 0, st0
    stream = torch.cuda.ExternalStream(g.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clk = ClockSampler(dev_index) if dev_index is not None else None
    if clk:
        clk.__enter__()
    with torch.cuda.stream(stream):
        e0.record(stream)
        st = g.step(steps)  # K graph launches, then the statistics (one small copy)
        e1.record(stream)
    torch.cuda.synchronize()
    if clk:
        clk.__exit__()
    assert st["status"] == 0, st
    out = g.download()
    if after:
        after(g)
    g.close()
    return e0.elapsed_time(e1), st, out, (clk.summary() if clk else None)


def _dump_timing(g, s):
    """Grid::printCols of the whole grid (device mark, download, parallel
    formatting, write) and the resume reader on that file, timed on the host."""
    import shutil
    import tempfile

    from gamma_b200 import gpu2d
    d = tempfile.mkdtemp(prefix="gamma_dump_")
    try:
        t0 = time.perf_counter()
        path = g.print_cols(d)
        t1 = time.perf_counter()
        nbytes = os.path.getsize(path)
        st, _, _ = gpu2d.text2d_read(path, s.ntheta, s.nmax)
        t2 = time.perf_counter()
        cells = int(sum(max(0, int(n) - 4) for n in st.ntrack[2:-2]))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return {"cells": cells, "bytes": nbytes, "write_s": t1 - t0, "read_s": t2 - t1,
            "write_cells_per_s": cells / (t1 - t0), "read_cells_per_s": cells / (t2 - t1),
            "host_threads": os.cpu_count()}


def _jet2d_ref_dump_worker(args):
    """The reference's own printCols and resume (libref_jet2d_io.so) on its 2D
    state after a few steps, timed."""
    params, warmup, root = args
    sys.path.insert(0, ROOT)
    os.makedirs(os.path.join(root, "results", "Last"), exist_ok=True)
    os.makedirs(os.path.join(root, "bin"), exist_ok=True)
    os.chdir(os.path.join(root, "bin"))
    from oracle.refsim2d import RefJet2D
    s = RefJet2D(io=True)
    s.set_params(**params)
    s.init()
    s.step(warmup)
    cells = sum(t.ntrack - 4 for t in s.snapshot().tracks[2:-2])
    t0 = time.perf_counter()
    s.print_cols()
    t1 = time.perf_counter()
    r = RefJet2D(io=True)
    r.set_params(**params)
    t2 = time.perf_counter()
    r.resume()  # reinitialise, updateGhosts and one more printCols
    t3 = time.perf_counter()
    return cells, t1 - t0, (t3 - t2) - (t1 - t0)


def _active_cells(out):
    o = np.arange(out.NJ) * out.cap
    return np.concatenate([np.arange(o[j] + 2, o[j] + int(out.ntrack[j]) - 2) for j in range(2, out.NJ - 2)])


def jet2d_arm(args, dev_index, host_work=True):
    """2D (r, theta) blast wave with a jet-like cap: 512 theta tracks over
    [0, 0.2] rad, BM profile (Gamma_shock^2 = 2e4) inside 0.1 rad, cold ambient
    outside, the reference problem module's regrid ratios (tracks settle at a
    few thousand cells), shock detection and synchrotron on.  Plain, then with
    the learned cons2prim start (trained on this run's states and drawn ones)
    from the same initial state, compared after the same steps."""
    from gamma_b200 import gpu, problems
    s = problems.Jet2dSetup(**dict(JET2D, ntheta=args.ntheta))
    dump = {}
    # host-side measurements (dump timing, CPU baselines) on one rank of one GPU only
    host_work = host_work and not args.no_cpu_baseline
    ms, st, out, clk = _jet2d_run(s, args.steps, args.warmup, 0, dev_index,
                                  after=None if (args.no_dump or not host_work)
                                  else (lambda g: dump.update(_dump_timing(g, s))))
    zones = st["zone_updates"]
    n = out.ntrack[2:-2]
    res = {"workload": f"{s.ntheta} theta tracks over [{s.th_min}, {s.th_max}] rad, BM cap below {s.th_jet} rad, "
                       f"{s.ncell} initial cells per track (reference regrid ratios), NUM_Q=10, regrid + shock "
                       "detection + synchrotron on",
           "value": zones / (ms / 1e3), "unit": "zone-updates/s", "ms_per_step": ms / args.steps,
           "zones_per_step": zones / args.steps, "cells_per_track": [int(n.min()), int(n.max())],
           "c2p": {"mean_newton_iters": st["c2p_iters"] / max(st["c2p_calls"], 1),
                   "max_newton_iters": st["c2p_max_iters"], "fallbacks": st["c2p_fallbacks"]},
           "clocks": clk, "gpu_launches": LAUNCHES_2D * args.steps}
    peak, peak_kind = measured_peak_hbm()
    achieved = B_ZU_NQ10 * zones / (ms / 1e3) / 1e9
    res["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "peak_source": peak_kind, "bytes_per_zone_update": B_ZU_NQ10,
                       "note": f"whole step ({LAUNCHES_2D} launches); per-kernel shares in the ncu launch list"}
    # the plain form: the same step with its kernels launched one by one (no
    # graph) and the reference's warm start, from the same initial state
    ms_p, st_p, out_p, _ = _jet2d_run(s, args.steps, args.warmup, 0, graphs=False)
    res["plain"] = {"value": st_p["zone_updates"] / (ms_p / 1e3), "ms_per_step": ms_p / args.steps,
                    "same_cell_counts": bool(np.array_equal(out_p.ntrack, out.ntrack)),
                    "note": f"{LAUNCHES_2D} kernel launches per step from the host, no CUDA graph, warm start"}
    res["batched_over_plain"] = res["value"] / res["plain"]["value"]
    if not args.no_learned:
        # training states: the run's active cells, as 1D states of the same |u| (cons2prim sees |S| only)
        live = _active_cells(out)
        prim = np.zeros((10, live.size))
        prim[:, :] = out.prim[:, live]
        prim[2] = np.hypot(out.prim[2, live], out.prim[3, live])
        prim[3] = 0.
        P, train = train_guess(gpu.config_sph(), prim, np.arange(live.size), SEED + 3)
        ms_l, st_l, out_l, _ = _jet2d_run(s, args.steps, args.warmup, P.data_ptr())
        same = bool(np.array_equal(out_l.ntrack, out.ntrack))
        l1 = None
        if same:
            l1 = {}
            for q, name in ((0, "rho"), (1, "p"), (2, "u_r"), (3, "u_theta"), (4, "tracer")):
                a, b = out_l.prim[q, live], out.prim[q, live]
                l1[name] = float(np.sum(np.abs(a - b)) / max(np.sum(np.abs(b)), 1e-300))
        res["learned_guess"] = {
            "value": st_l["zone_updates"] / (ms_l / 1e3), "unit": "zone-updates/s", "ms_per_step": ms_l / args.steps,
            "mean_newton_iters": st_l["c2p_iters"] / max(st_l["c2p_calls"], 1),
            "max_newton_iters": st_l["c2p_max_iters"], "fallbacks": st_l["c2p_fallbacks"],
            "fallback_rate": st_l["c2p_fallbacks"] / max(st_l["c2p_calls"], 1),
            "guess_rate": st_l["c2p_guesses"] / max(st_l["c2p_calls"], 1),
            "poor_warm_start_rate": st_l["c2p_poor"] / max(st_l["c2p_calls"], 1),
            "steps_with_guess": st_l["learned_steps"], "steps_timed": args.steps,
            "plain_mean_newton_iters": res["c2p"]["mean_newton_iters"],
            "plain_max_newton_iters": res["c2p"]["max_newton_iters"],
            "same_cell_counts": same, "l1_vs_plain": l1, "steps_compared": max(args.warmup, 3) + 1 + args.steps,
            "training": train,
            "note": GATE_NOTE + " (guess_rate); regrid merges keep the warm start; Newton still converges to the "
                    "reference tolerance"}
        res["learned_over_plain"] = res["learned_guess"]["value"] / res["plain"]["value"]
        del P
    lib = os.path.join(ROOT, "oracle", "_ref", "libref_jet2d.so")
    if host_work and os.path.exists(lib):
        import multiprocessing as mp
        # a 16-track wedge with 1,200 initial cells per track (the reference moves
        # whole Cell records for every merge, so its first regrid grows with the
        # square of the track length; per-zone step cost does not), single-threaded:
        # its 2D flux loop accumulates into neighbour cells from several threads
        p = dict(ncell=1200, ntrack=16, nmax=1200)
        with mp.get_context("spawn").Pool(1) as pool:
            z, t = pool.apply(_jet2d_cpu_worker, ((p, 10, 3),))
        res["cpu_baseline"] = {"value": z / t, "unit": "zone-updates/s", "cores": 1, "kind": "reference",
                               "sample": "the same wedge with 16 tracks of 1,200 initial cells, 10 steps after 3 "
                                         "warm-up steps, one thread"}
    if host_work and os.path.exists(lib.replace("jet2d.so", "jet2d_io.so")):
        import multiprocessing as mp
        import shutil
        import tempfile
        root = tempfile.mkdtemp(prefix="gamma_refdump_")
        try:
            with mp.get_context("spawn").Pool(1) as pool:
                cells, tw, tr = pool.apply(_jet2d_ref_dump_worker, ((dict(ncell=1200, ntrack=16, nmax=1200), 3,
                                                                     root),))
        finally:
            shutil.rmtree(root, ignore_errors=True)
        dump["reference"] = {"cells": cells, "write_cells_per_s": cells / tw, "read_cells_per_s": cells / max(tr, 1e-9),
                             "note": "the reference's printCols / reinitialise on the 16-track wedge, one thread; "
                                     "its read time is the resume minus one printCols"}
    if dump:
        res["dump"] = dump
    return res


def jet2d_c4_arm(args, dev_index):
    """The sweep workload's large 2D case: 4,096 theta tracks of ~8,000 cells
    over [0, 0.2] rad (~33 M zones), the jet set-up of the 2D workload, batched
    (one graph per step), device-resident."""
    import torch

    from gamma_b200 import problems
    s = problems.Jet2dSetup(**dict(JET2D_C4, ntheta=args.c4_ntheta))
    free0 = torch.cuda.mem_get_info()[0]
    mem = []
    ms, st, out, clk = _jet2d_run(s, args.steps, args.warmup, 0, dev_index,
                                  after=lambda g: mem.append(torch.cuda.mem_get_info()[0]))
    zones = st["zone_updates"]
    n = out.ntrack[2:-2]
    peak, peak_kind = measured_peak_hbm()
    achieved = B_ZU_NQ10 * zones / (ms / 1e3) / 1e9
    return {"workload": f"{s.ntheta} theta tracks over [{s.th_min}, {s.th_max}] rad, BM cap below {s.th_jet} rad, "
                        f"{s.ncell} initial cells per track, slow cells merged below {s.merge_DR_slow} of the target "
                        "spacing, NUM_Q=10, regrid + shock detection + synchrotron on",
            "value": zones / (ms / 1e3), "unit": "zone-updates/s", "ms_per_step": ms / args.steps,
            "zones_per_step": zones / args.steps, "cells_per_track": [int(n.min()), int(n.max())],
            "device_state_gb": (free0 - mem[0]) / 1e9 if mem else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "bytes_per_zone_update": B_ZU_NQ10},
            "clocks": clk, "gpu_launches": LAUNCHES_2D * args.steps}


def summary_of(line):
    """Short top-level figures of every workload, placed last in the JSON line."""
    def get(d, *path):
        for k in path:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    def r(v):
        return None if v is None else float(f"{v:.4g}")
    out = {"tubes_value": get(line, "value"), "tubes_e2e": get(line, "e2e", "value"),
           "tubes_frac": get(line, "roofline", "frac"), "tubes_learned_value": get(line, "learned_guess", "value")}
    for w in ("jet2d", "sweep"):
        out[f"{w}_value"] = get(line, w, "value")
        out[f"{w}_plain_value"] = get(line, w, "plain", "value")
        out[f"{w}_learned_value"] = get(line, w, "learned_guess", "value")
        out[f"{w}_batched_over_plain"] = get(line, w, "batched_over_plain")
        out[f"{w}_learned_over_plain"] = get(line, w, "learned_over_plain")
        out[f"{w}_learned_guess_rate"] = get(line, w, "learned_guess", "guess_rate")
        lv, bv = out[f"{w}_learned_value"], out[f"{w}_value"]
        out[f"{w}_learned_over_batched"] = lv / bv if lv and bv else None
        out[f"{w}_frac"] = get(line, w, "roofline", "frac")
    out["c4_2d_value"] = get(line, "sweep2d", "value")
    out["c4_2d_zones_per_step"] = get(line, "sweep2d", "zones_per_step")
    out["c4_2d_frac"] = get(line, "sweep2d", "roofline", "frac")
    out["c2p_plain_value"] = get(line, "c2p", "plain", "value")
    out["c2p_learned_value"] = get(line, "c2p", "learned", "value")
    out["c2p_learned_over_plain"] = get(line, "c2p", "speedup_learned")
    tl = out["tubes_learned_value"]
    out["tubes_learned_over_batched"] = tl / out["tubes_value"] if tl and out["tubes_value"] else None
    return {k: r(v) for k, v in out.items() if v is not None}


def autotune(g, args):
    """The step kernel's launch shape picked on the live state (gamma_gpu_autotune:
    3 one-step launches per shape, state restored), outside the timed region."""
    from gamma_b200 import gpu
    if args.variant is not None:
        g.set_variant(args.variant)
        th, cpt = gpu.variant_info(args.variant)
        return {"threads": th, "cells_per_thread": cpt, "tuned": False}
    if args.no_tune:
        return {"threads": 128, "cells_per_thread": 1, "tuned": False}
    ms, v = g.autotune(3)
    th, cpt = gpu.variant_info(v)
    return {"threads": th, "cells_per_thread": cpt, "tuned": True,
            "ms_per_3_steps": {f"{a}x{b}": round(m, 3) for m, (a, b) in
                               zip(ms, (gpu.variant_info(k) for k in range(gpu.N_VARIANTS)))}}


GATE_NOTE = ("a step runs the kernel with the network only if the previous step found poor warm starts (first "
             "Newton correction above 3% of the previous pressure) in more than a quarter of its cons2prim calls "
             "(steps_with_guess of steps_timed); there, cells with a poor warm start search again from the network's "
             "pressure")

TRAIN_PAIRS = 10_000_000  # the learned guess's training set (half from solution states where there are enough)


def train_guess(cfg, prim, rows_live, seed):
    """Train the learned cons2prim starting pressure on device.

    Training pairs: 10 M, half of them (or all the run has, if fewer) primitive
    states picked from the columns `rows_live` of `prim` [nq][N] (host array),
    the rest drawn.  Returns the device parameter tensor and a summary."""
    import torch

    from gamma_b200 import gpu
    dev = torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(rows_live, size=min(TRAIN_PAIRS // 2, rows_live.size), replace=False))
    states = torch.tensor(np.ascontiguousarray(prim[:, pick]), device=dev)
    ns = states.shape[1]
    nu = TRAIN_PAIRS - ns
    x = torch.zeros((ns + nu, 3), dtype=torch.float32, device=dev)
    y = torch.zeros((ns + nu, 2), dtype=torch.float32, device=dev)
    gpu.mlp_pairs(cfg, states.data_ptr(), ns, nu, seed, x.data_ptr(), y.data_ptr())
    P = torch.zeros(gpu.mlp_param_count(), dtype=torch.float32, device=dev)
    gpu.mlp_init(P.data_ptr(), seed)
    loss = gpu.mlp_train(P.data_ptr(), x.data_ptr(), y.data_ptr(), ns + nu, epochs=6, batch=8192)
    torch.cuda.synchronize()
    return P, {"pairs": ns + nu, "from_states": ns, "drawn": nu, "epochs": len(loss),
               "final_loss": float(loss[-1]), "seconds": time.perf_counter() - t0}


def live_cells(offsets, ntrack):
    return np.concatenate([np.arange(o, o + n) for o, n in zip(offsets, ntrack)])


def l1_live(got, want, offsets, ntrack, rows):
    """max over `rows` of the L1 relative difference over the active cells of every run."""
    act = np.concatenate([np.arange(o + 2, o + n - 2) for o, n in zip(offsets, ntrack)])
    return max(float(np.sum(np.abs(got[q, act] - want[q, act])) / max(np.sum(np.abs(want[q, act])), 1e-300))
               for q in rows)


def learned_arm(args, g, cfg, upload, stream, plain_out, rows, max_over_ranks, barrier, ws, plain_stats):
    """The same workload with the learned cons2prim starting pressure.

    The network is trained here (training pairs: up to 1M states of the runs
    after the plain arm's steps plus 1M drawn states); the result after K steps
    from the initial state is compared with the plain run's (L1 over the active
    cells and stored slots; every run must keep the plain run's cell count)."""
    import torch

    out = g.download()
    P, train = train_guess(cfg, out["prim"], live_cells(g.offsets, out["ntrack"]), SEED)
    g.set_guess(P.data_ptr())
    # the launch shape of the step with the guess, tuned like the plain step's
    plain_variant = g.variant
    tune = autotune(g, args)
    # results: K steps from the initial state, against the plain run's K steps
    upload()
    g.step(args.steps, stats=False)
    got = g.download()
    same = bool(np.array_equal(got["ntrack"], plain_out["ntrack"]))
    l1 = l1_live(got["prim"], plain_out["prim"], g.offsets, plain_out["ntrack"], rows) if same else None
    # timing: same protocol as the plain arm
    upload()
    for _ in range(args.warmup):
        g.step(1, stats=False)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    zones = learned = poor = calls = 0
    barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for k in range(args.steps):
            s1 = g.step(1)
            zones += s1["zone_updates"]
            learned += s1["learned_steps"]
            poor += s1["c2p_poor"]
            calls += s1["c2p_calls"]
            ev[k + 1].record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(sum(ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)))
    st = g.step(1)
    g.set_guess(0)
    g.set_variant(plain_variant)
    return {
        "value": ws * zones / (ms / 1e3), "unit": "zone-updates/s", "ms_per_step": ms / args.steps,
        "mean_newton_iters": st["c2p_iters"] / max(st["c2p_calls"], 1), "max_newton_iters": st["c2p_max_iters"],
        "fallbacks": st["c2p_fallbacks"], "fallback_rate": st["c2p_fallbacks"] / max(st["c2p_calls"], 1),
        "guess_rate": st["c2p_guesses"] / max(st["c2p_calls"], 1),
        "poor_warm_start_rate": poor / max(calls, 1), "steps_with_guess": learned, "steps_timed": args.steps,
        "plain_mean_newton_iters": plain_stats["c2p_iters"] / max(plain_stats["c2p_calls"], 1),
        "l1_vs_plain": l1, "same_cell_counts": same, "steps_compared": args.steps, "training": train,
        "launch_shape": tune,
        "note": GATE_NOTE + " (guess_rate of the calls); Newton still converges to the reference tolerance",
    }


C2P_STATES = 1 << 24


def c2p_states(n, seed=SEED):
    """Seeded spherical-hydro states (NUM_Q = 10) over the learned guess's
    training range: Lorentz factor log-uniform in [1, 1e3], p/rho in
    [1e-10, 1e3], rho in [1e-6, 1e6]; their conserved variables (the
    FluidState::prim2cons formulas, ideal gas, Gamma = 4/3, written out here)."""
    rng = np.random.default_rng(seed + 5)
    lfac = np.exp(rng.uniform(0., np.log(1e3), n))
    rho = 10. ** rng.uniform(-6., 6., n)
    p = rho * 10. ** rng.uniform(-10., 3., n)
    u = np.sqrt(lfac * lfac - 1.) * rng.choice([-1., 1.], n)
    prim = np.zeros((10, n))
    prim[0], prim[1], prim[2], prim[4] = rho, p, u, 1.
    G = 4. / 3.
    h = 1. + p * G / (G - 1.) / rho
    D = lfac * rho
    cons = np.zeros((10, n))
    cons[0], cons[1], cons[2], cons[4] = D, D * h * lfac - p - D, D * h * u, D
    return prim, cons


def _c2p_cpu_worker(args):
    """The reference's own FluidState::cons2prim (GSL Brent through the shim) on
    a slice of the states, from the same cold start."""
    cons, prim0 = args
    sys.path.insert(0, ROOT)
    from oracle.refsim import RefSim
    s = RefSim("bm1d")
    t0 = time.perf_counter()
    s.cons2prim(cons, prim0)
    return cons.shape[1], time.perf_counter() - t0


def c2p_arm(args, dev_index, host_work=True):
    """FluidState::cons2prim on a batch of 16.8 M independent states with no
    previous pressure (the start is p = 1): the plain Newton from that start,
    and Newton from the learned guess (BF16 tensor-core inference fused into
    the kernel), against each other and the reference's CPU routine."""
    import torch

    from gamma_b200 import gpu
    n = args.c2p_states
    prim, cons = c2p_states(n)
    cold = prim.copy()
    cold[1] = 1.
    cfg = gpu.config_sph()
    dev = torch.device("cuda", dev_index)
    dcons0 = torch.tensor(cons, device=dev)
    dcold = torch.tensor(cold, device=dev)
    it = torch.zeros(n, dtype=torch.int32, device=dev)
    # the network, trained on drawn states of the same range
    nu = 2_000_000
    x = torch.zeros((nu, 3), dtype=torch.float32, device=dev)
    y = torch.zeros((nu, 2), dtype=torch.float32, device=dev)
    gpu.mlp_pairs(cfg, 0, 0, nu, SEED + 6, x.data_ptr(), y.data_ptr())
    P = torch.zeros(gpu.mlp_param_count(), dtype=torch.float32, device=dev)
    gpu.mlp_init(P.data_ptr(), SEED)
    t0 = time.perf_counter()
    loss = gpu.mlp_train(P.data_ptr(), x.data_ptr(), y.data_ptr(), nu, epochs=6, batch=8192)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    res = {"workload": f"{n} independent spherical-hydro states (NUM_Q=10, Gamma=4/3), Lorentz factor log-uniform "
                       "in [1,1e3], p/rho in [1e-10,1e3], rho in [1e-6,1e6]; cons2prim from p = 1",
           "states": n, "unit": "states/s"}
    out = {}
    for name in ("plain", "learned"):
        times = []
        for k in range(max(args.warmup, 3) + args.steps):
            dcons = dcons0.clone()
            dprim = dcold.clone()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            if name == "plain":
                gpu.cons2prim_device(cfg, dcons.data_ptr(), dprim.data_ptr(), n, it.data_ptr())
            else:
                gpu.cons2prim_guess_device(cfg, dcons.data_ptr(), dprim.data_ptr(), n, P.data_ptr(), it.data_ptr())
            e1.record()
            torch.cuda.synchronize()
            if k >= max(args.warmup, 3):
                times.append(e0.elapsed_time(e1))
        iters = it.cpu().numpy()
        out[name] = dprim.cpu().numpy()
        ms = statistics.mean(times)
        res[name] = {"value": n / (ms / 1e3), "ms": ms, "mean_newton_iters": float(iters.mean()),
                     "max_newton_iters": int(iters.max()), "fallback_rate": float(np.mean(iters > 100))}
        # per state: cons and the prim guess read, prim and the rewritten cons written
        achieved = 4 * 10 * 8 * n / (ms / 1e3) / 1e9
        peak, kind = measured_peak_hbm()
        res[name]["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                 "frac": achieved / peak, "peak_source": kind, "bytes_per_state": 320}
    for q, nm in ((0, "rho"), (1, "p"), (2, "u")):
        a, b = out["learned"][q], out["plain"][q]
        res.setdefault("l1_learned_vs_plain", {})[nm] = float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))
    res["speedup_learned"] = res["learned"]["value"] / res["plain"]["value"]
    res["training"] = {"pairs": nu, "epochs": len(loss), "final_loss": float(loss[-1]), "seconds": train_s}
    if host_work and not args.no_cpu_baseline and os.path.exists(os.path.join(ROOT, "oracle", "_ref",
                                                                              "libref_bm1d.so")):
        import multiprocessing as mp
        cores = os.cpu_count() or 1
        m = 40_000 * cores
        chunks = [(np.ascontiguousarray(cons[:, k:m:cores]), np.ascontiguousarray(cold[:, k:m:cores]))
                  for k in range(cores)]
        with mp.get_context("spawn").Pool(cores) as pool:
            r = pool.map(_c2p_cpu_worker, chunks)
        res["cpu_baseline"] = {"value": sum(a for a, _ in r) / max(t for _, t in r), "unit": "states/s",
                               "cores": cores, "kind": "reference",
                               "sample": f"the first {m} states, one process per core, from the same start"}
    return res


SWEEP_RUNS = 1024


def sweep_setups(nruns=SWEEP_RUNS, seed=SEED):
    """Parameter sweep of BM1D blast waves: log10 E_iso ~ U(50, 54) erg,
    log10 n ~ U(-3, 1) cm^-3, N ~ U{1000..8000} log-spaced cells over
    [0.9, 1.1] R_shock, Gamma_shock = 100, nmax = 2N."""
    rng = np.random.default_rng(seed + 1)
    E = 10. ** rng.uniform(50., 54., nruns)
    n = 10. ** rng.uniform(-3., 1., nruns)
    N = rng.integers(1000, 8001, nruns)
    return [dict(eta=1e-10, lorentz_mode=1, lfac_shock2=1e4, Etot=float(E[i]), n_ext=float(n[i]), ncell=int(N[i]),
                 nmax=2 * int(N[i]), grid_log=1, r_lo=0.9, r_hi=1.1) for i in range(nruns)]


def _sweep_init(kws):
    sys.path.insert(0, ROOT)
    from gamma_b200 import problems
    return [problems.Bm1dSetup(**kw).initial_state() for kw in kws]


def _sweep_cpu_worker(args):
    """The reference's own BM1D build (oracle/_ref/libref_bm1d.so) on some of the
    sweep's runs: zone-updates of the timed steps and their seconds."""
    kws, steps, warmup = args
    sys.path.insert(0, ROOT)
    from oracle.refsim import RefSim
    zones, busy = 0, 0.0
    for kw in kws:  # one process-wide Simu per library: re-initialised per run
        s = RefSim("bm1d")
        s.set_params(**kw)
        s.init()
        s.step(warmup)
        for _ in range(steps):
            t0 = time.perf_counter()
            s.step(1)
            busy += time.perf_counter() - t0
            zones += int(s.scalars()["nact"])
    return zones, busy


def sweep_cpu_baseline(kws, cores, warmup, steps=3):
    import multiprocessing as mp
    rng = np.random.default_rng(SEED + 2)
    idx = rng.choice(len(kws), size=min(2 * cores, len(kws)), replace=False)
    sample = [kws[i] for i in idx]
    chunks = [sample[k::cores] for k in range(cores)]
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_sweep_cpu_worker, [(ch, steps, warmup) for ch in chunks if ch])
    zones = sum(r[0] for r in res)
    value = zones / max(r[1] for r in res)
    return {"value": value, "unit": "zone-updates/s", "cores": cores, "kind": "reference",
            "sample": f"{len(sample)} of the {len(kws)} runs (seeded), {steps} timed steps each after {warmup} "
                      f"warm-up steps, {cores} processes; value = sample zone-updates / slowest process"}


def sweep_plain(args, kws, states):
    """The plain drop-in form of the sweep: every run in a context of its own
    (one Simu each, as separate GAMMA jobs would be), default launch shape, no
    CUDA graph, no tuner, warm start.  A step is one gamma_gpu_step per
    context, each on its context's own stream.  The same steps from the same
    initial states as the batched arm: warm-up, one more, then K timed, which
    take the same zone-updates (checked through the final cell counts)."""
    import torch

    from gamma_b200 import gpu, problems
    cfg = gpu.config_sph()
    ctxs = []
    for kw, st in zip(kws, states):
        s = problems.Bm1dSetup(**kw)
        g = gpu.GammaGPU(cfg, [s.capacity])
        g.set_params([s.run_params()])
        g.use_graphs(False)
        pk = problems.pack([st], g.offsets, g.total, 10)
        g.upload(pk["ntrack"], pk["prim"], pk["x"], pk["dx"], pk["xI"], pk["dt_loc"], pk["t"], pk["it"])
        ctxs.append(g)
    for _ in range(max(args.warmup, 3) + 1):
        for g in ctxs:
            g.step(1, stats=False)
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    streams = [torch.cuda.ExternalStream(g.stream) for g in ctxs]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ends = [torch.cuda.Event() for _ in ctxs]
    e0.record(side)
    for st in streams:
        st.wait_event(e0)
    for _ in range(args.steps):
        for g in ctxs:
            g.step(1, stats=False)
    for ev, st in zip(ends, streams):
        ev.record(st)
    for ev in ends:
        side.wait_event(ev)
    e1.record(side)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    nt = np.array([int(g.download()["ntrack"][0]) for g in ctxs])
    for g in ctxs:
        g.close()
    return ms, nt


def sweep_arm(args, dev_index, max_over_ranks, barrier, ws):
    """C4: independent BM1D runs of uneven size and parameters, one persistent
    launch per step (one CTA per run, work queue longest-first), regrid, shock
    detection and synchrotron on; plain and with the learned guess."""
    import multiprocessing as mp

    import torch

    from gamma_b200 import gpu, problems
    kws = sweep_setups(args.sweep_runs)
    setups = [problems.Bm1dSetup(**k) for k in kws]
    chunks = [kws[i::16] for i in range(16)]
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        parts = pool.map(_sweep_init, chunks)
    states = [None] * len(kws)
    for i in range(16):
        states[i::16] = parts[i]
    cfg = gpu.config_sph()
    g = gpu.GammaGPU(cfg, [s.capacity for s in setups])
    g.set_params([s.run_params() for s in setups])
    pk = problems.pack(states, g.offsets, g.total, 10)
    host = {k: torch.from_numpy(np.ascontiguousarray(pk[k])).pin_memory() for k in ("prim", "x", "dx", "dt_loc", "xI")}
    out_prim = torch.empty_like(host["prim"]).pin_memory()
    stream = torch.cuda.ExternalStream(g.stream)

    def upload():
        g.upload_ptrs(pk["ntrack"], pk["t"], pk["it"], host["prim"].data_ptr(), host["x"].data_ptr(),
                      host["dx"].data_ptr(), host["dt_loc"].data_ptr(), host["xI"].data_ptr())

    upload()
    for _ in range(max(args.warmup, 3)):
        g.step(1, stats=False)
    tune = autotune(g, args)
    stats0 = g.step(1)
    assert stats0["status"] == 0, stats0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    zones = 0
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev_index) as clk:
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            for k in range(args.steps):
                zones += g.step(1)["zone_updates"]
                ev[k + 1].record(stream)
        torch.cuda.synchronize()
    barrier()
    per_launch = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    ms = max_over_ranks(sum(per_launch))
    nt_timed = g.download()["ntrack"].copy()
    # end to end from pinned host memory: upload, K steps, download of the
    # primitives.  These K steps start from the initial state, whose first
    # regrids merge most cells one run at a time and want many resident runs,
    # so the launch shape is tuned again on that state (outside the region).
    upload()
    tune_e2e = autotune(g, args)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    zones_e2e = 0
    barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0.record(stream)
        upload()
        for _ in range(args.steps):
            zones_e2e += g.step(1)["zone_updates"]
        nt_e2e = g.download_ptrs(out_prim.data_ptr())
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    plain_out = {"ntrack": nt_e2e, "prim": out_prim.numpy().copy()}
    peak, peak_kind = measured_peak_hbm()
    achieved = B_ZU_NQ10 * (zones / args.steps) / (statistics.mean(per_launch) / 1e3) / 1e9
    res = {"workload": f"{len(kws)} BM1D blast waves (spherical, Gamma=4/3, NUM_Q=10), log10 E_iso ~ U(50,54), "
                       "log10 n ~ U(-3,1), N ~ U{1000..8000} log-spaced cells over [0.9,1.1] R_shock, "
                       "Gamma_shock=100, nmax=2N; regrid + shock detection + synchrotron on; one RK3 step of "
                       "every run per launch",
           "runs": len(kws), "initial_zones": int(sum(k["ncell"] for k in kws)),
           "value": ws * zones / (ms / 1e3), "unit": "zone-updates/s", "ms_per_step": ms / args.steps,
           "zones_per_step": zones / args.steps,
           "e2e": {"value": ws * zones_e2e / (e2e_ms / 1e3), "unit": "zone-updates/s",
                   "h2d_bytes_per_step": (sum(v.numel() * 8 for v in host.values()) - host["prim"].numel() * 8 // 10)
                   / args.steps, "d2h_bytes_per_step": out_prim.numel() * 8 * 9 // 10 / args.steps},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_source": peak_kind, "bytes_per_zone_update": B_ZU_NQ10},
           "c2p": {"mean_newton_iters": stats0["c2p_iters"] / max(stats0["c2p_calls"], 1),
                   "max_newton_iters": stats0["c2p_max_iters"], "fallbacks": stats0["c2p_fallbacks"]},
           "regrid_per_step": {"splits": stats0["splits"], "merges": stats0["merges"]},
           "clocks": clk.summary(), "gpu_launches": args.steps, "launch_shape": tune,
           "launch_shape_e2e": tune_e2e}
    if not args.no_learned:
        res["learned_guess"] = learned_arm(args, g, cfg, upload, stream, plain_out, (0, 1, 2, 4, 5, 6, 7, 8, 9),
                                           max_over_ranks, barrier, ws, stats0)
    g.close()
    if not args.no_plain:
        ms_p, nt_p = sweep_plain(args, kws, states)
        ms_p = max_over_ranks(ms_p)
        res["plain"] = {"value": ws * zones / (ms_p / 1e3), "ms_per_step": ms_p / args.steps,
                        "same_cell_counts": bool(np.array_equal(nt_p, nt_timed)),
                        "note": "one context per run (1,024 gamma_gpu_step calls per step, each one CTA on its "
                                "own stream), default launch shape, no graph, no tuner"}
        res["batched_over_plain"] = res["value"] / res["plain"]["value"]
        if "learned_guess" in res:
            res["learned_over_plain"] = res["learned_guess"]["value"] / res["plain"]["value"]
    if not args.no_cpu_baseline and ws == 1 and os.path.exists(os.path.join(ROOT, "oracle", "_ref",
                                                                            "libref_bm1d.so")):
        res["cpu_baseline"] = sweep_cpu_baseline(kws, os.cpu_count() or 1, max(args.warmup, 3))
    return res


def rank_sync(ws, device):
    """Replicas only: the ranks share no data, only a barrier around each timed
    region and the slowest rank's time (all-reduce MAX)."""
    import torch

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if ws == 1:
            return x
        t = torch.tensor([x], device=device, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())
    return barrier, max_over_ranks


def run_gpu_arm(args):
    import torch

    from gamma_b200 import gpu, problems

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    barrier, max_over_ranks = rank_sync(ws, "cuda")

    if args.workload != "all":  # one workload alone, as its own line (profiling captures)
        if args.workload == "jet2d":
            res = jet2d_arm(args, local)
        elif args.workload == "sweep":
            res = sweep_arm(args, local, max_over_ranks, barrier, ws)
        elif args.workload == "c2p":
            res = c2p_arm(args, local)
        elif args.workload == "sweep2d":
            res = jet2d_c4_arm(args, local)
        if args.workload != "tubes":
            if rank == 0:
                print(json.dumps(dict({"metric": METRIC, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                                       "higher_is_better": True, "dtype": "f64", "data": "synthetic"}, **res)))
            if ws > 1:
                torch.distributed.destroy_process_group()
            return

    setups = tube_setups(args.ntubes)
    states = [s.initial_state() for s in setups]
    g = gpu.GammaGPU(gpu.config_cart(), [s.capacity for s in setups])
    pk = problems.pack(states, g.offsets, g.total, 6)
    zones_per_step = sum(s.ncell for s in setups)

    # pinned host buffers for the end-to-end arm
    host = {k: torch.from_numpy(np.ascontiguousarray(pk[k])).pin_memory() for k in ("prim", "x", "dx", "dt_loc", "xI")}
    out_prim = torch.empty_like(host["prim"]).pin_memory()
    h2d_bytes = sum(v.numel() * 8 for k, v in host.items()) - host["prim"].numel() * 8 // 6  # slot 3 is not sent
    d2h_bytes = out_prim.numel() * 8 * 5 // 6

    def upload():
        g.upload_ptrs(pk["ntrack"], pk["t"], pk["it"], host["prim"].data_ptr(), host["x"].data_ptr(),
                      host["dx"].data_ptr(), host["dt_loc"].data_ptr(), host["xI"].data_ptr())

    stream = torch.cuda.ExternalStream(g.stream)

    upload()
    for _ in range(args.warmup):
        g.step(1, stats=False)
    tune = autotune(g, args)
    torch.cuda.synchronize()
    stats0 = g.step(1)  # one step with statistics, outside the timed region
    assert stats0["status"] == 0, stats0

    # ---- device-resident timing: K launches, one RK3 step each
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            for k in range(args.steps):
                g.step(1, stats=False)
                ev[k + 1].record(stream)
        torch.cuda.synchronize()
    barrier()
    per_launch = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    ms_total = max_over_ranks(sum(per_launch))
    ms_step = ms_total / args.steps
    value = ws * zones_per_step * args.steps / (ms_total / 1e3)

    # ---- end to end through the C ABI from pinned host memory: upload, K steps, download
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        upload()
        for _ in range(args.steps):
            g.step(1, stats=False)
        nt_e2e = g.download_ptrs(out_prim.data_ptr())
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = ws * zones_per_step * args.steps / (e2e_ms / 1e3)

    peak, peak_kind = measured_peak_hbm()
    achieved = B_ZU_NQ6 * zones_per_step / (statistics.mean(per_launch) / 1e3) / 1e9
    tz = traffic_per_zone()
    line = {
        "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.ntubes} cartesian relativistic shock tubes, 256-8192 cells (log-uniform), "
                               "Gamma=5/3, NUM_Q=6, one RK3 step of every tube per launch", "tubes": args.ntubes,
                   "zones_per_step": zones_per_step, "seed": SEED, "l2": "state 1.4 GB > L2 (no flush needed)",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU"},
        "e2e": {"value": e2e_value, "unit": "zone-updates/s", "h2d_bytes_per_step": h2d_bytes / args.steps,
                "d2h_bytes_per_step": d2h_bytes / args.steps,
                "definition": "pinned-host upload of the initial state, K steps, download of the final "
                              "primitives, through gamma_gpu_upload/step/download"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "bytes_per_zone_update": B_ZU_NQ6,
                     "traffic": None if tz is None else tz * zones_per_step},
        "clocks": clk.summary(),
        "gpu_launches": args.steps,
        "launch_shape": tune,
        "c2p": {"mean_newton_iters": stats0["c2p_iters"] / max(stats0["c2p_calls"], 1),
                "max_newton_iters": stats0["c2p_max_iters"], "fallbacks": stats0["c2p_fallbacks"]},
    }
    if not args.no_learned:
        line["learned_guess"] = learned_arm(args, g, gpu.config_cart(), upload, stream,
                                            {"ntrack": nt_e2e, "prim": out_prim.numpy().copy()}, (0, 1, 2, 4, 5),
                                            max_over_ranks, barrier, ws, stats0)
    g.close()
    if not args.no_2d and args.workload == "all":
        line["jet2d"] = jet2d_arm(args, local, host_work=(ws == 1 and rank == 0))
    if not args.no_sweep and args.workload == "all":
        line["sweep"] = sweep_arm(args, local, max_over_ranks, barrier, ws)
    if not args.no_c4_2d and args.workload == "all":
        line["sweep2d"] = jet2d_c4_arm(args, local)
    if not args.no_c2p and args.workload == "all" and rank == 0:
        line["c2p"] = c2p_arm(args, local, host_work=(ws == 1))
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        setups_cpu = setups
        cores = os.cpu_count() or 1
        v, info, _ = cpu_run(setups_cpu, 50, 2, sample=max(64, cores * 2), cores=cores,
                             budget_zones=float(os.environ.get("GAMMA_CPU_ZONES", 3.0e7)))
        line["cpu_baseline"] = dict(info, value=v, unit="zone-updates/s")
    line["summary"] = summary_of(line)
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gamma", choices=["gamma", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned cons2prim guess arm")
    ap.add_argument("--no-2d", action="store_true", help="skip the 2D (r, theta) workload")
    ap.add_argument("--no-sweep", action="store_true", help="skip the BM1D parameter sweep")
    ap.add_argument("--no-dump", action="store_true", help="skip the 2D text dump and resume timing")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shape of the 1D step")
    ap.add_argument("--variant", type=int, default=None, help="a fixed launch shape of the 1D step (no tuning)")
    ap.add_argument("--workload", default="all", choices=["all", "tubes", "jet2d", "sweep", "sweep2d", "c2p"],
                    help="one workload alone (profiling captures); 'all' prints the tube line with the others nested")
    ap.add_argument("--ntubes", type=int, default=NTUBES, help="smaller batches for profiling captures")
    ap.add_argument("--ntheta", type=int, default=JET2D["ntheta"], help="theta tracks of the 2D workload")
    ap.add_argument("--sweep-runs", type=int, default=SWEEP_RUNS, help="runs of the BM1D sweep")
    ap.add_argument("--c2p-states", type=int, default=C2P_STATES, help="states of the cons2prim batch")
    ap.add_argument("--no-c2p", action="store_true", help="skip the cons2prim batch")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain (one context per run) sweep arm")
    ap.add_argument("--no-c4-2d", action="store_true", help="skip the large 2D case of the sweep workload")
    ap.add_argument("--c4-ntheta", type=int, default=JET2D_C4["ntheta"], help="theta tracks of the large 2D case")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
