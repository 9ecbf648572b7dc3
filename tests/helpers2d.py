"""2D parity helpers: the reference's snapshots in the C ABI's layout, and
the comparison metrics of the 2D tests."""
import numpy as np

NQ = 10


def state_from_reference(snap):
    """A State2D holding a reference snapshot (oracle.refsim2d.Grid2D),
    including the fields the reference carries between stages."""
    from gamma_b200.gpu2d import State2D
    NJ, cap = len(snap.tracks), snap.cap
    NC = NJ * cap
    prim, gmv, gf1 = np.zeros((NQ, NC)), np.zeros((NQ, NC)), np.zeros((NQ, NC))
    x, dx, xI = np.zeros(NC), np.zeros(NC), np.zeros(NC)
    dtl = np.full(NC, 1e15)
    nbr = np.zeros((4, NC), np.int32)
    nbr[0] = nbr[2] = -1
    for j, t in enumerate(snap.tracks):
        o, n = j * cap, t.ntrack
        prim[:, o:o + n] = t.prim
        gmv[:, o:o + n] = t.grad_mv
        gf1[:, o:o + n] = t.grad_f1
        x[o:o + n], dx[o:o + n], dtl[o:o + n] = t.x, t.dx, t.dt_loc
        xI[o:o + n - 1] = t.xI
        nbr[0, o:o + n], nbr[1, o:o + n] = t.nbr[:, 0, 0], t.nbr[:, 0, 1]
        nbr[2, o:o + n], nbr[3, o:o + n] = t.nbr[:, 1, 0], t.nbr[:, 1, 1]
    nt = np.array([t.ntrack for t in snap.tracks], np.int32)
    return State2D(NJ, cap, nt, prim, x, dx, xI, dtl, gmv, gf1, nbr, snap.t, snap.it)


def theta_of(snap, ngst=2):
    act = snap.tracks[ngst:len(snap.tracks) - ngst]
    return np.array([t.th[ngst] for t in act]), np.array([t.dth[ngst] for t in act])


def params_of(p, derived):
    """gamma_2d_params_t of a jet2d parameter set (defaults of the problem module)"""
    import math

    from gamma_b200.gpu2d import Params2D
    MP, ME, ALPHA = 1.6726219e-24, 9.1093835e-28, 1.29251816e-09
    rhoN, vN, lN = derived["rhoNorm"], derived["vNorm"], derived["lNorm"]
    return Params2D(p.get("split_DR", 5.), p.get("merge_DR", 0.3), p.get("split_DR_slow", 20.),
                    p.get("merge_DR_slow", 1.2), p.get("v_out", 1.05), p.get("it_hold", 1000.),
                    ALPHA / (1. / (rhoN * vN * lN)), MP / (rhoN * math.pow(lN, 3)), ME / (rhoN * math.pow(lN, 3)))


def energy(prim, gamma_ad=4. / 3.):
    lf = np.sqrt(1 + prim[2] ** 2 + prim[3] ** 2)
    h = 1 + gamma_ad / (gamma_ad - 1) * prim[1] / prim[0]
    return prim[0] * lf * lf * h - prim[1]


def active_pairs(got, ref, ngst=2):
    """(track index, got track dict, reference track) of the active tracks"""
    for j in range(ngst, len(ref.tracks) - ngst):
        yield j, got.track(j), ref.tracks[j]


def l1_by_quantity(got, ref, qs=(0, 1, 2, 3, 4, 6, 7, 9), ngst=2):
    out = {}
    for q in qs:
        num = den = 0.
        for _, a, b in active_pairs(got, ref, ngst):
            s = slice(ngst, b.ntrack - ngst)
            num += np.sum(np.abs(a["prim"][q][s] - b.prim[q][s]))
            den += np.sum(np.abs(b.prim[q][s]))
        out[q] = num / den if den > 0 else num
    return out


def l1_between_snapshots(a, b, qs, ngst=2):
    """L1 of reference snapshot a against reference snapshot b (the same cell
    counts), per quantity, over the active cells of the active tracks"""
    out = {}
    for q in qs:
        num = den = 0.
        for j in range(ngst, len(b.tracks) - ngst):
            s = slice(ngst, b.tracks[j].ntrack - ngst)
            num += np.sum(np.abs(a.tracks[j].prim[q][s] - b.tracks[j].prim[q][s]))
            den += np.sum(np.abs(b.tracks[j].prim[q][s]))
        out[q] = num / den if den > 0 else num
    return out


def cell_errors(got, ref, q, ngst=2):
    """relative errors of quantity q over the active cells: pressures against
    max(|p|, 1e-2 E), velocities with a floor of 1e-6 of their largest value"""
    errs = []
    umax = max(np.max(np.abs(t.prim[q])) for t in ref.tracks[ngst:-ngst]) if q in (2, 3) else 0.
    for _, a, b in active_pairs(got, ref, ngst):
        s = slice(ngst, b.ntrack - ngst)
        va, vb = a["prim"][q][s], b.prim[q][s]
        if q == 1:
            floor = 1e-2 * energy(b.prim)[s]
        elif q in (2, 3):
            floor = np.full_like(vb, 1e-6 * umax + 1e-300)
        else:
            floor = np.full_like(vb, 1e-300)
        errs.append(np.abs(va - vb) / np.maximum(np.abs(vb), floor))
    return np.concatenate(errs)
