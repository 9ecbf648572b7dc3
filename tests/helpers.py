"""Comparison helpers shared by the parity tests."""
import numpy as np

# Fields of a track snapshot and the slots compared (slot 3 is zero in 1D).
PRIM_NAMES = {0: "rho", 1: "p", 2: "u", 3: "u_theta", 4: "tracer1", 5: "tracer2", 6: "gamma_min",
              7: "gamma_max", 8: "gamma_mid", 9: "p_syn"}


def energy_scale(prim, gamma_ad):
    """E = D + tau of each cell: the scale to which cons2prim determines p.

    The pressure is the root of f(p) = E + p - D lfac - k p lfac^2; rounding in
    f is a few ulp of E, so p itself is only defined to ~eps * E / |f'(p)|.  In a
    cold cell (p/rho ~ 1e-10) that is ~1e-6 of p, for the reference's own Brent
    solver as much as for Newton, so pressure-like errors are measured against E.
    """
    rho, p, u = prim[0], prim[1], prim[2]
    lfac = np.sqrt(1.0 + u * u)
    h = 1.0 + p * gamma_ad / (gamma_ad - 1.0) / rho
    return rho * lfac * h * lfac - p


EPS = 2.220446049250313e-16
# f(p) = E + p - D lfac - k p lfac^2 is rounded to a few ulp of E, so where p
# is far below E (cold gas) any root finder leaves p uncertain by ~eps * E:
# pressures are held to max(rtol |p|, P_EPS_E * eps * E)
P_EPS_E = 16.0


def pressure_scale(p, E, rtol):
    """The scale s with |dp| <= rtol * s  <=>  |dp| <= max(rtol |p|, P_EPS_E eps E)."""
    return np.maximum(np.abs(p), P_EPS_E * EPS * np.abs(E) / rtol)


def rel_err(a, b, floor):
    """max |a-b| / max(|b|, floor)"""
    d = np.abs(a - b) / np.maximum(np.abs(b), floor)
    return float(np.max(d)) if d.size else 0.0


def compare_track(gpu, ref, gamma_ad, nq, rtol, etol=None):
    """Per-field relative errors of a GPU track vs the oracle track.

    rtol applies to every primitive and to x, dx, xI; the pressure (and the
    tracers that follow it) use floor etol * E (see energy_scale)."""
    assert gpu.ntrack == ref.ntrack, (gpu.ntrack, ref.ntrack)
    E = energy_scale(ref.prim, gamma_ad)
    errs = {}
    for q in range(nq):
        if q == 3:
            continue
        a, b = gpu.prim[q], ref.prim[q]
        if q == 1 and etol is not None:
            floor = etol * E
        else:
            floor = np.full_like(b, 1e-300)
        errs[PRIM_NAMES[q]] = rel_err(a, b, floor)
    errs["x"] = rel_err(gpu.x, ref.x, 1e-300)
    errs["dx"] = rel_err(gpu.dx, ref.dx, 1e-300)
    errs["xI"] = rel_err(gpu.xI, ref.xI, 1e-300)
    return errs


def l1_rel(a, b):
    """sum |a-b| / sum |b| over active cells"""
    den = np.sum(np.abs(b))
    return float(np.sum(np.abs(a - b)) / den) if den > 0 else float(np.sum(np.abs(a - b)))


def solver_sensitivity(run, eps_list=(1e-13, 1e-14, 1e-15), converged=1e-16):
    """How much the oracle's own solution moves when only its pressure root
    finder stops elsewhere.

    run(eps) returns an oracle snapshot after the same steps with Brent
    stopping at relative bracket eps.  Returns (converged snapshot, per-field
    per-cell max |snap(eps) - snap(converged)| over eps_list)."""
    ref = run(converged)
    sens = {}
    for eps in eps_list:
        s = run(eps)
        assert s.ntrack == ref.ntrack
        for q in range(ref.prim.shape[0]):
            d = np.abs(s.prim[q] - ref.prim[q])
            sens[q] = np.maximum(sens.get(q, 0.0), d)
    return ref, sens


def within_sensitivity(got, ref, sens, gamma_ad, rtol=1e-12, k=4.0, qs=(0, 1, 2)):
    """Per-cell check |got - ref| <= rtol * scale + k * sensitivity.

    scale is |ref| (pressure: pressure_scale, i.e. rtol * scale is at least
    P_EPS_E eps E).  Returns the worst ratio
    |got - ref| / bound per field (<= 1 passes) and the fraction of cells that
    are within rtol alone."""
    E = energy_scale(ref.prim, gamma_ad)
    worst, frac = {}, {}
    for q in qs:
        b = ref.prim[q]
        scale = pressure_scale(b, E, rtol) if q == 1 else np.abs(b)
        if q >= 2:
            # velocities and tracers vanish in parts of a track: below 1e-4 of
            # the field's largest magnitude (or of one for a track at rest)
            # differences are rounding of the fluxes that carry them
            scale = np.maximum(scale, 1e-4 * max(np.max(np.abs(b)), 1.0 if q == 2 else 1e-300))
        d = np.abs(got.prim[q] - b)
        bound = rtol * scale + k * sens[q]
        worst[q] = float(np.max(d / np.maximum(bound, 1e-300)))
        frac[q] = float(np.mean(d <= rtol * scale))
    return worst, frac


def record(quantity, measured, bar, better="lower"):
    """Append one measured parity figure to $GAMMA_PARITY_RECORD (JSON lines).

    Tests call this before asserting, so a run over several builds (arithmetic
    forms, FMA contraction) yields a table of what each build measures against
    each bar, failures included.  Without the variable it does nothing."""
    import json
    import os
    path = os.environ.get("GAMMA_PARITY_RECORD")
    if not path:
        return
    test = os.environ.get("PYTEST_CURRENT_TEST", "?").split(" ")[0]
    with open(path, "a") as f:
        f.write(json.dumps({"test": test, "quantity": quantity, "measured": float(measured), "bar": float(bar),
                            "better": better, "lib": os.environ.get("GAMMA_B200_LIB", "default")}) + "\n")
