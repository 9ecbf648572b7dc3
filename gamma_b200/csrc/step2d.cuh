// The 2D (r, theta) moving-mesh step of GAMMA as per-element functions.
//
// A run is a set of NJ theta tracks (ngst ghost tracks on each side), each a
// 1D moving mesh in r of at most `cap` cells (ghosts included).  Cell (j, i)
// lives at flat index g = j * cap + i, which is also the reference's cell id
// (Cell::nde_id, src/Dimensions/2d.cpp:100-106), so the neighbour lists can be
// stored as (first id, count).  Interface (j, i) is the right edge of cell
// (j, i).  Per step (src/simu.cpp:79-105, src/Timestep/rk3.cpp:98-194):
//
//   regrid (per track) -> [reset shocks] -> per stage:
//     ghosts            updateGhosts (2d.cpp:241-321)
//     mv_interface      reconstructStates(MV) + computeLambda + kinematics +
//                       computeFlux + measureShock (2d.cpp:436-470, 735-767)
//     cell_mv           update_dt(MV) and computeNeighbors (2d.cpp:534-606, 769-777)
//     trans_grad        computeTransGradients (2d.cpp:366-430)
//     f1_if/f1_gather   the theta-direction fluxes between tracks (2d.cpp:779-839)
//     [stage 1: dt = CFL min dt_loc, detectShock]
//     iface_move, update_cell   Grid::update + the RK3 combines (2d.cpp:861-882,
//                       rk3.cpp:98-194)
//   -> inject particles.
// With the Euler module (src/Timestep/euler.cpp:12-19) there is one stage and
// no combine.
//
// Fields the reference keeps in its Cell records across stages and steps are
// kept here too, because they feed later results: the moving-direction and
// transverse gradients (grad_mv, grad_f1) and the neighbour lists.  In the
// reference the ghost cells 0 and ntrack-1 of each track are copies of an edge
// cell made before the neighbour lists are rebuilt, so they use the lists and
// gradients of an earlier stage (and, in ghost tracks, lists that point into
// other tracks); the transverse gradient of the upper cell of a theta
// interface is the one from the previous stage (track j+1 is processed after
// track j).  Each of these is reproduced.
#pragma once

#include "physics2d.cuh"
#include "search.cuh"

namespace gb {
namespace d2 {

constexpr int KMAX_STALE = 8;  // foreign stale contributors per target track
// a theta interface's results: flux[NQ], forward Sd, reverse Sd, flags (1: the
// forward test reached the spectral index, 2: the reverse one)
constexpr int IF_WORDS = NQ + 3;

// Problem hooks of the theta-wedge blast wave (src/Initial/Tests/BM.cpp)
struct Params2 {
  double split_DR, merge_DR;            // checkCellForRegrid ratios for lfac >= 2
  double split_DR_slow, merge_DR_slow;  // ... and for lfac < 2
  double v_out;                         // outer ghost-interface velocity
  double it_hold;                       // v_out -> 0 once it > it_hold and the flow has stopped
  double Nalpha, Nmp, Nme;              // synchrotron constants (normalised)
};

struct Grid2 {
  int NJ, cap, ngst;
  long long NC;  // NJ * cap: row stride of [q][g] arrays
  int *ntrack;   // [NJ]
  const double *tg;  // [NJ][TG_WORDS] angular factors of each track (TrackGeo)
  // cells
  double *prim;       // [NQ][NC]
  double *x, *dx;     // r and dr (Cell::G)
  double *dtl, *sd, *pspec;
  uint8_t *shocked;
  double *gmv, *gf1, *gf1n;  // [NQ][NC] grad_mv, grad_f1 (persistent), grad_f1 of this stage
  int *nbr;                  // [4][NC]: first id and count towards track j-1, then j+1
  double *cons0, *dV0;       // [NQ][NC], [NC]: S0.cons and G0.dV (copyState0)
  double *f1lo, *f1hi;       // [NQ][NC]: flux[0][F1], flux[1][F1]
  // interfaces
  double *xI, *xI0, *xIm;    // position, step-start position, position after the stage's move
  double *v, *lL, *lR;
  double *flx;               // [NQ][NC] MV flux (times dA)
  // foreign stale contributors: stale_n[t], stale_id[t * KMAX_STALE + k]
  int *stale_n, *stale_id;
  // run scalars
  double *t, *dt;
  long long *it;
  int *status;               // 30: negative CFL candidate; 40: stale table overflow;
                             // 41: a track's theta interfaces exceed if_cap
  double *red;               // partial minima of dt_loc
  int *pref;                 // [NJ+1] cells of tracks before j (the live-cell index)
  int *gtrk;                 // [NC/32+2] track of live cell 32k (k_group_tracks)
  // theta interfaces, owned by the cells of track j (j <= NJ-2) through their
  // upper lists, numbered per track in cell order (k_if_scan):
  double *ifs;               // [IF_WORDS][NJ * if_cap]: interface results, track j from j * if_cap
  int *if_off;               // [NC]: a cell's first interface within its track
  int *if_own;               // [NJ * if_cap]: the owning cell (index in its track) of each interface
  int *if_tot;               // [NJ]: interfaces of each track
  int *if_pref;              // [NJ+1]: interfaces of the tracks before j
  int *iftrk;                // [(NJ-1) if_cap/32 + 2] track of interface 32k (k_if_group_tracks)
  // regrid scratch (one track of records per track)
  double *rprim, *rgmv, *rgf1;  // [NQ][NC]
  double *rx, *rdx, *rdtl, *rxI;
  int *rnbr;                 // [4][NC]
  double *rdV;               // [NC] new cells' right interface (original index, or -1)
  int *rseg;                 // [2 NC]: per track, cap segment starts then cap sources
  int *rnbr2;                // [4][NC]
  unsigned long long *stats;  // c2p calls, c2p iters, fallbacks, zone updates, splits, merges, max iters
};

// interfaces one track may own: its upper lists overlap the next track's
// cells in sorted order, so they hold at most ntrack[j] + ntrack[j+1] entries;
// the margin covers the copied lists of the edge cells
__host__ __device__ inline long long if_cap(const Grid2 &G) { return 2LL * G.cap + 64; }

GB_HD int iL_of(const Grid2 &G) { return G.ngst - 1; }
GB_HD int jL_of(const Grid2 &G) { return G.ngst - 1; }
GB_HD int jR_of(const Grid2 &G) { return G.NJ - G.ngst; }

GB_HD double cen_r(double r, double dr) {
  double r2 = r * r;
  double dr2 = dr * dr;
  return 3. * r * (r2 + dr2) / (3 * r2 + dr2);
}

GB_HD TrackGeo tgeo(const Grid2 &G, int j) { return track_geo(G.tg + (long long)j * TG_WORDS); }

GB_HD Geom cell_geom(const Grid2 &G, int j, long long g) { return make_geom(G.x[g], G.dx[g], tgeo(G, j)); }

GB_HD void load_prim(const Grid2 &G, long long g, double *p) {
#pragma unroll
  for (int q = 0; q < NQ; ++q) p[q] = G.prim[q * G.NC + g];
}

// ---------------------------------------------------------------------------
// Ghost tracks and ghost cells (Grid::updateGhosts, 2d.cpp:241-321).  One
// track per call, threads tid of nth.  `reset`: the step's first call, right
// after Cell::resetShock of every cell.  The source cells of a ghost track are
// never written in the same pass (only active cells are copied).

// All loads are issued before the first store: the arrays are distinct, but
// the compiler cannot prove it and would otherwise wait on each load in turn.
GB_HD void copy_cell(const Grid2 &G, long long d, long long s, bool reset) {
  double p[NQ], gm[NQ], gf[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    p[q] = G.prim[q * G.NC + s];
    gm[q] = G.gmv[q * G.NC + s];
    gf[q] = G.gf1[q * G.NC + s];
  }
  const double x = G.x[s], dx = G.dx[s], dtl = G.dtl[s];
  double sd = -1., ps = 0.;
  int sh = 0;
  if (!reset) {
    sd = G.sd[s];
    ps = G.pspec[s];
    sh = G.shocked[s];
  }
  int nb[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) nb[k] = G.nbr[k * G.NC + s];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    G.prim[q * G.NC + d] = p[q];
    G.gmv[q * G.NC + d] = gm[q];
    G.gf1[q * G.NC + d] = gf[q];
  }
  G.x[d] = x;
  G.dx[d] = dx;
  G.dtl[d] = dtl;
  G.sd[d] = sd;
  G.pspec[d] = ps;
  G.shocked[d] = sh;
#pragma unroll
  for (int k = 0; k < 4; ++k) G.nbr[k * G.NC + d] = nb[k];
}

// track holding the pooled cell id g (ids fit in int: NC < 2^31 is checked at creation)
GB_HD int track_of(const Grid2 &G, long long g) { return (int)g / G.cap; }

// phase 1: a ghost track takes the active cells and interfaces of the edge
// track; slot i of ghost track number k (0..2 ngst-1, lower tracks first)
GB_HD int ghost_track(const Grid2 &G, int k) { return k < G.ngst ? k : G.NJ - 2 * G.ngst + k; }

GB_HD void ghosts_track_slot(const Grid2 &G, int k, int i, bool reset) {
  const int j = ghost_track(G, k);
  const int src = j <= jL_of(G) ? jL_of(G) + 1 : jR_of(G) - 1;
  const int n = G.ntrack[src];
  const int iL = iL_of(G), iR = n - G.ngst;
  if (i == 0) G.ntrack[j] = n;
  const long long o = (long long)j * G.cap, os = (long long)src * G.cap;
  if (i >= iL + 1 && i <= iR - 1) copy_cell(G, o + i, os + i, reset);
  if (i >= iL && i <= iR - 1) G.xI[o + i] = G.xI[os + i];
}

// phase 2: ghost cells and ghost interfaces of the track (after phase 1)
GB_HD void ghosts_cells(const Grid2 &G, int j, int tid, int nth) {
  const int n = G.ntrack[j];
  const int iL = iL_of(G), iR = n - G.ngst;
  const long long o = (long long)j * G.cap;
  const long long eL = o + iL + 1, eR = o + iR - 1;
  for (int i = tid; i <= iL; i += nth) {
    copy_cell(G, o + i, eL, false);
    G.x[o + i] = G.x[eL] - (iL - i + 1) * G.dx[eL];
  }
  for (int i = iR + tid; i < n; i += nth) {
    copy_cell(G, o + i, eR, false);
    G.x[o + i] = G.x[eR] + (i - iR + 1) * G.dx[eR];
  }
  for (int i = tid; i <= iL - 1; i += nth) G.xI[o + i] = G.xI[o + iL + 1] - (iL - i + 1) * G.dx[eL];
  for (int i = iR + tid; i <= n - 2; i += nth) G.xI[o + i] = G.xI[o + iR - 1] + (i - iR) * G.dx[eR];
}

// ---------------------------------------------------------------------------
// Moving-direction interfaces (one per call): reconstructStates(MV),
// computeLambda, updateKinematics + userKinematics, computeFlux, measureShock.

// userKinematics of BM.cpp:198-218: the outer ghost interfaces move at v_out
// until, after it_hold steps, the flow ten cells inside the outer edge of the
// first active track has stopped.
GB_HD double outer_velocity(const Grid2 &G, const Params2 &P, long long it) {
  const int jt = jL_of(G) + 1;
  const int iR = G.ntrack[jt] - G.ngst;
  const long long g = (long long)jt * G.cap + iR - 10;
  if (G.prim[UU1 * G.NC + g] < 1.e-3 && (double)it > P.it_hold) return 0.;
  return P.v_out;
}

// cell state as prepForUpdate leaves it: prim2cons and state2flux at the cell's r
GB_HD void cell_state(const Phys &ph, const Grid2 &G, long long g, int dim, St &S) {
  load_prim(G, g, S.prim);
  fill(ph, S, dim, G.x[g]);
}

GB_HD void mv_interface(const Phys &ph, const Params2 &P, const Grid2 &G, int j, int i, long long it) {
  const int n = G.ntrack[j];
  if (i > n - 2) return;
  const long long o = (long long)j * G.cap, g = o + i;
  const double xI = G.xI[g];
  St L, R;
  if (i == 0 || i == n - 2) {
    cell_state(ph, G, g, MV, L);
    cell_state(ph, G, g + 1, MV, R);
  } else {
    const double cLL = cen_r(G.x[g - 1], G.dx[g - 1]), cL = cen_r(G.x[g], G.dx[g]);
    const double cR = cen_r(G.x[g + 1], G.dx[g + 1]), cRR = cen_r(G.x[g + 2], G.dx[g + 2]);
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const double qLL = G.prim[q * G.NC + g - 1], qL = G.prim[q * G.NC + g];
      const double qR = G.prim[q * G.NC + g + 1], qRR = G.prim[q * G.NC + g + 2];
      double gL = qdiv(qL - qLL, cL - cLL);
      const double gN = qdiv(qR - qL, cR - cL);
      double gR = qdiv(qRR - qR, cRR - cR);
      gL = minmod(gL, gN);
      gR = minmod(gR, gN);
      // grad_mv stored in the cells; cell i from its right interface, except
      // the last reconstructed cell n-2, which only has its left one
      G.gmv[q * G.NC + g] = gL;
      if (i == n - 3) G.gmv[q * G.NC + g + 1] = gR;
      L.prim[q] = qL + gL * (xI - cL);
      R.prim[q] = qR + gR * (xI - cR);
    }
    fill(ph, L, MV, xI);
    fill(ph, R, MV, xI);
  }
  const Waves w = compute_lambda(ph, L, R, MV, xI);
  double v = ph.vi * w.lS;
  if (i >= n - 1 - G.ngst) v = outer_velocity(G, P, it);
  G.lL[g] = w.lL;
  G.lR[g] = w.lR;
  G.v[g] = v;
  double fl[NQ];
  hllc_flux(L, R, w, v, dA_r(xI, tgeo(G, j)), MV, xI, fl);
#pragma unroll
  for (int q = 0; q < NQ; ++q) G.flx[q * G.NC + g] = fl[q];
  // measureShock, moving direction: forward shocks only, into the left cell
  double Sd;
  if (compute_Sd(ph, sd_side(L, MV), sd_side(R, MV), false, &Sd)) {
    if (P_SPEC > G.pspec[g]) G.pspec[g] = P_SPEC;
  }
  G.sd[g] = fmax(G.sd[g], Sd);
}

// ---------------------------------------------------------------------------
// Per cell after the interfaces: update_dt(MV) (cell.cpp:47-74) and the
// neighbour lists (computeNeighbors, 2d.cpp:534-606) of cells 1..ntrack-2.
//
// The reference scans the interfaces of track j-/+1 with a cursor carried from
// cell to cell.  With those interfaces sorted, the cursor at the start of cell
// i is min(LB(x_{i-1} + dx_{i-1}/2), n'-2) (LB: first interface >= the value),
// which gives every list without the scan.

GB_HD void neighbour_list(const Grid2 &G, int j, int i, int jn, int *first, int *count) {
  const long long o = (long long)j * G.cap, g = o + i;
  const int np = G.ntrack[jn];
  const double *X = G.xI + (long long)jn * G.cap;  // np-1 interfaces
  const double xjL = G.x[g] - G.dx[g] / 2.;
  const double xjR = G.x[g] + G.dx[g] / 2.;
  int s = 0;
  if (i > 1) {
    // LB(xpR), from the start of this list in the previous stage (nbr still
    // holds it; a regrid or an upload only makes the hint worse)
    const double xpR = G.x[g - 1] + G.dx[g - 1] / 2.;
    const long long hint = (long long)G.nbr[(jn < j ? 0 : 2) * G.NC + g] - (long long)jn * G.cap;
    s = partition_from(0, np - 1, hint, [&](int k) { return X[k] < xpR; });
    if (s > np - 2) s = np - 2;
  }
  const int b = (X[s] > xjL && s > 0) ? s - 1 : s;
  if (X[b] < xjR) {
    // LB(xjR) - 1: with X[b] < xjR and X sorted, LB(xjR) > b, so a scan from
    // b + 1 finds it in (list length + 1) loads
    int e = b + 1;
    while (e < np - 1 && X[e] < xjR) ++e;
    --e;
    if (e > np - 2) e = np - 2;
    *first = jn * G.cap + b + 1;
    *count = e - b + 1;
  } else {
    *first = jn * G.cap + b + 1;  // empty: kept ordered for the gather's search
    *count = 0;
  }
}

GB_HD void cell_mv(const Grid2 &G, int j, int i) {
  const int n = G.ntrack[j];
  if (i < 1 || i > n - 2) return;
  const long long g = (long long)j * G.cap + i;
  // Cell::update_dt, moving direction
  const double a = G.dx[g];
  double dL = (G.lR[g - 1] > G.v[g]) ? a / (G.lR[g - 1] - G.v[g]) : DT_INF;
  double dR = (G.lL[g] < G.v[g - 1]) ? a / (G.v[g - 1] - G.lL[g]) : DT_INF;
  const double cand = fmin(dL, dR);
  if (cand < 0) *G.status = 30;
  else G.dtl[g] = fmin(G.dtl[g], cand);
  // neighbour lists
  int f0 = -1, c0 = 0, f1 = -1, c1 = 0;
  if (j != 0) neighbour_list(G, j, i, j - 1, &f0, &c0);
  if (j != G.NJ - 1) neighbour_list(G, j, i, j + 1, &f1, &c1);
  G.nbr[0 * G.NC + g] = f0;
  G.nbr[1 * G.NC + g] = c0;
  G.nbr[2 * G.NC + g] = f1;
  G.nbr[3 * G.NC + g] = c1;
}

// ---------------------------------------------------------------------------
// Transverse gradient of cell (j, i), j <= NJ-2 (computeTransGradients).
// The theta position of the interface with an upper neighbour stays at the
// cell centre there (the reference's `else if (d==0)` never moves it).

GB_HD void overlap(const Grid2 &G, long long g0, long long gn, double *xm, double *w) {
  const double xL0 = G.x[g0] - G.dx[g0] / 2., xR0 = G.x[g0] + G.dx[g0] / 2.;
  const double xLn = G.x[gn] - G.dx[gn] / 2., xRn = G.x[gn] + G.dx[gn] / 2.;
  *xm = (fmax(xL0, xLn) + fmin(xR0, xRn)) / 2.;
  *w = fmax(0., fmin(xR0, xRn) - fmax(xL0, xLn));
}

// Geometry of the gradient towards neighbour gn, the same for every slot:
// the offsets of the overlap's centre from both cell centres, the theta
// distance, and the overlap's area.
struct NbrGeo {
  double dxmL, dxmR, dcen, dA;
};

GB_HD NbrGeo neighbour_geo(const Grid2 &G, long long g0, long long gn, double cr0, double ct0, double s) {
  double xm, w;
  overlap(G, g0, gn, &xm, &w);
  NbrGeo n;
  n.dxmL = xm - cr0;
  n.dxmR = xm - cen_r(G.x[gn], G.dx[gn]);
  n.dcen = tgeo(G, track_of(G, gn)).cen_t - ct0;
  n.dA = dA_t(xm, w, s);
  return n;
}

// The gradient of slot q towards neighbour gn, (qR - qL) / dcen.
GB_HD double neighbour_grad(const Grid2 &G, int q, long long gn, const NbrGeo &n, double p0, double m0) {
  const double qL = p0 + m0 * n.dxmL;
  const double qR = G.prim[q * G.NC + gn] + G.gmv[q * G.NC + gn] * n.dxmR;
  return qdiv(qR - qL, n.dcen);
}

// Pass 1 forms the dA-weighted average; pass 2 folds in minmod with each
// neighbour's gradient in the reference's order (an order-dependent chain:
// minmod(x, x) = 0).  Every slot's chain uses its own gradients only, so the
// slots run one after another over geometry formed once: the first KGEO
// neighbours' geometry and one slot's gradients stay in registers, and
// neighbours past KGEO recompute theirs for each slot.  Per slot the
// operations and their order are those of the reference's loops.
constexpr int KGEO = 4;

GB_HD void trans_grad(const Grid2 &G, int j, int i) {
  const int n = G.ntrack[j];
  if (i >= n) return;
  const long long g0 = (long long)j * G.cap + i;
  if (j == G.NJ - 1) {  // never recomputed: keeps its copied value
#pragma unroll
    for (int q = 0; q < NQ; ++q) G.gf1n[q * G.NC + g0] = G.gf1[q * G.NC + g0];
    return;
  }
  const double cr0 = cen_r(G.x[g0], G.dx[g0]);
  const TrackGeo t0 = tgeo(G, j);
  const double ct0 = t0.cen_t;
  const int f0 = G.nbr[0 * G.NC + g0], c0 = G.nbr[1 * G.NC + g0];
  const int f1 = G.nbr[2 * G.NC + g0], c1 = G.nbr[3 * G.NC + g0];
  const int nn = c0 + c1;
  // neighbour kn: the lower list's cells, then the upper list's; the theta of
  // the interface is th - dth/2 below and th (unmoved) above
#define TG_NBR(kn) ((kn) < c0 ? (long long)f0 + (kn) : (long long)f1 + ((kn) - c0))
#define TG_S(kn) ((kn) < c0 ? t0.s_lo : t0.s_mid)
  NbrGeo geo[KGEO];
  double dAtot = 0.;
#pragma unroll
  for (int kn = 0; kn < KGEO; ++kn)
    if (kn < nn) {
      geo[kn] = neighbour_geo(G, g0, TG_NBR(kn), cr0, ct0, TG_S(kn));
      dAtot += geo[kn].dA;
    }
  for (int kn = KGEO; kn < nn; ++kn) dAtot += neighbour_geo(G, g0, TG_NBR(kn), cr0, ct0, TG_S(kn)).dA;
#pragma unroll 1
  for (int q = 0; q < NQ; ++q) {
    const double p0 = G.prim[q * G.NC + g0], m0 = G.gmv[q * G.NC + g0];
    double avg = 0., kept[KGEO];
#pragma unroll
    for (int kn = 0; kn < KGEO; ++kn)
      if (kn < nn) {
        kept[kn] = neighbour_grad(G, q, TG_NBR(kn), geo[kn], p0, m0);
        avg += kept[kn] * geo[kn].dA;
      }
    for (int kn = KGEO; kn < nn; ++kn) {
      const NbrGeo e = neighbour_geo(G, g0, TG_NBR(kn), cr0, ct0, TG_S(kn));
      avg += neighbour_grad(G, q, TG_NBR(kn), e, p0, m0) * e.dA;
    }
    avg = qdiv(avg, dAtot);
#pragma unroll
    for (int kn = 0; kn < KGEO; ++kn)
      if (kn < nn) avg = minmod(avg, kept[kn]);
    for (int kn = KGEO; kn < nn; ++kn) {
      const NbrGeo e = neighbour_geo(G, g0, TG_NBR(kn), cr0, ct0, TG_S(kn));
      avg = minmod(avg, neighbour_grad(G, q, TG_NBR(kn), e, p0, m0));
    }
    G.gf1n[q * G.NC + g0] = avg;
  }
#undef TG_NBR
#undef TG_S
}

// ---------------------------------------------------------------------------
// Theta-direction interface between c0 = (j, i) and its upper neighbour gn
// (the body of the F1 loop of Grid::computeFluxes, 2d.cpp:800-837).

struct F1Result {
  double flux[NQ];
  double sd_fwd, sd_rev;
  bool have_fwd, have_rev;
};

GB_HD void f1_interface(const Phys &ph, const Grid2 &G, int j, long long g0, long long gn, F1Result &out) {
  const int jn = track_of(G, gn);
  const TrackGeo t0 = tgeo(G, j);
  const double jpos = t0.th + t0.dth / 2.;
  double xm, w;
  overlap(G, g0, gn, &xm, &w);
  const double dA = dA_t(xm, w, t0.s_hi);
  St L, R;
  const bool pc = j == 0 || j == G.NJ - 2 || G.nbr[1 * G.NC + g0] == 0 || G.nbr[3 * G.NC + gn] == 0;
  if (pc) {
    cell_state(ph, G, g0, F1, L);
    cell_state(ph, G, gn, F1, R);
  } else {
    // the upper cell's transverse gradient: this stage's if the reference's
    // track-by-track loop has reached it already, else the previous stage's
    const double *gR = (jn < j || (jn == j && gn < g0)) ? G.gf1n : G.gf1;
    const double dxmL = xm - cen_r(G.x[g0], G.dx[g0]);
    const double dxmR = xm - cen_r(G.x[gn], G.dx[gn]);
    const double dxfL = jpos - t0.cen_t;
    const double dxfR = jpos - tgeo(G, jn).cen_t;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const double qL = G.prim[q * G.NC + g0] + G.gmv[q * G.NC + g0] * dxmL;
      const double qR = G.prim[q * G.NC + gn] + G.gmv[q * G.NC + gn] * dxmR;
      L.prim[q] = qL + G.gf1n[q * G.NC + g0] * dxfL;  // this stage's (computed first)
      R.prim[q] = qR + gR[q * G.NC + gn] * dxfR;
    }
    fill(ph, L, F1, xm);
    fill(ph, R, F1, xm);
  }
  const Waves wv = compute_lambda(ph, L, R, F1, xm);
  hllc_flux(L, R, wv, 0., dA, F1, xm, out.flux);
  // measureShock across the tracks (radiation_sph.cpp:160-175): the forward
  // test (L upstream) and the reverse one (R upstream).  compute_Sd passes its
  // pressure test only where the upstream pressure is the larger, so at most
  // one of the two evaluates the isentrope integral: one call, with the
  // upstream side chosen per lane, gives both results and runs the integral
  // once per warp instead of twice.  Where a pressure is NaN both tests pass
  // and both results are NaN, which the one call also gives.
  const SdSide sL = sd_side(L, F1), sR = sd_side(R, F1);
  const bool fw = sL.p > sR.p;
  const bool nan_p = isnan(sL.p) || isnan(sR.p);
  double sd;
  const bool have = compute_Sd(ph, fw ? sL : sR, fw ? sR : sL, !fw, &sd);
  out.have_fwd = (fw || nan_p) && have;
  out.sd_fwd = (fw || nan_p) ? sd : -1.;
  out.have_rev = !fw && have;
  out.sd_rev = fw ? -1. : sd;
}

// Interface s of track j's list: upper neighbour k of its owning cell.  Its
// flux, shock tests and flags are kept for the cell pass (f1_gather).  One
// interface per thread: a cell's upper list holds one to three of them, and a
// thread per cell left the lanes of the shorter lists idle.
GB_HD void f1_if(const Phys &ph, const Grid2 &G, int j, int s) {
  const long long base = (long long)j * if_cap(G), sl = base + s;
  const long long g0 = (long long)j * G.cap + G.if_own[sl];
  const int k = s - G.if_off[g0];
  F1Result r;
  f1_interface(ph, G, j, g0, G.nbr[2 * G.NC + g0] + k, r);
  const long long IS = (long long)G.NJ * if_cap(G);
#pragma unroll
  for (int q = 0; q < NQ; ++q) G.ifs[q * IS + sl] = r.flux[q];
  G.ifs[NQ * IS + sl] = r.sd_fwd;
  G.ifs[(NQ + 1) * IS + sl] = r.sd_rev;
  G.ifs[(NQ + 2) * IS + sl] = (r.have_fwd ? 1. : 0.) + (r.have_rev ? 2. : 0.);
}

// Foreign stale contributors: cells 0 and ntrack-1 whose (copied) upper list
// points into a track other than j+1.  Each track appends its own (stale_n
// cleared first); the gather puts a target's entries in (j, i) order.
GB_HD void stale_append(const Grid2 &G, int j) {
  const int n = G.ntrack[j];
  const int cells[2] = {0, n - 1};
  for (int c = 0; c < 2; ++c) {
    const long long g = (long long)j * G.cap + cells[c];
    const int first = G.nbr[2 * G.NC + g], cnt = G.nbr[3 * G.NC + g];
    if (cnt <= 0) continue;
    const int t = track_of(G, first);
    if (t == j + 1 || t < 0 || t >= G.NJ) continue;
#ifdef __CUDA_ARCH__
    const int k = atomicAdd(&G.stale_n[t], 1);
#else
    const int k = G.stale_n[t]++;
#endif
    if (k >= KMAX_STALE) {
      *G.status = 40;
      continue;
    }
    G.stale_id[t * KMAX_STALE + k] = (int)g;
  }
}

GB_HD void stale_table(const Grid2 &G) {
  for (int t = 0; t < G.NJ; ++t) G.stale_n[t] = 0;
  for (int j = 0; j <= G.NJ - 2; ++j) stale_append(G, j);
}

// Cell cn after f1_if: its own side (flux[1][F1], forward shocks over its
// upper list) and its other side (flux[0][F1] and reverse shocks, summed over
// the cells whose upper list holds cn, in the reference's (j, i) order).
GB_HD void f1_gather(const Phys &ph, const Grid2 &G, int t, int k) {
  (void)ph;
  if (k >= G.ntrack[t]) return;
  const long long gn = (long long)t * G.cap + k;
  const long long IC = if_cap(G), IS = (long long)G.NJ * IC;
  double sd = G.sd[gn], ps = G.pspec[gn];
  // the cell's own side: flux[1][F1] and the forward shock tests over its
  // upper list, in order (tracks 0..NJ-2)
  if (t <= G.NJ - 2) {
    const int cnt = G.nbr[3 * G.NC + gn], off = G.if_off[gn];
    const long long sl0 = (long long)t * IC + off;
    double hi[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) hi[q] = 0.;
    for (int m = 0; m < cnt && off + m < IC; ++m) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) hi[q] += G.ifs[q * IS + sl0 + m];
      sd = fmax(sd, G.ifs[NQ * IS + sl0 + m]);
      if (((int)G.ifs[(NQ + 2) * IS + sl0 + m] & 1) && P_SPEC > ps) ps = P_SPEC;
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) G.f1hi[q * G.NC + gn] = hi[q];
  }
  double acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) acc[q] = 0.;
  auto add = [&](int j, long long g0) {
    const int first = G.nbr[2 * G.NC + g0], cnt = G.nbr[3 * G.NC + g0];
    if (!(cnt > 0 && gn >= first && gn < (long long)first + cnt)) return;
    const long long s = G.if_off[g0] + (gn - first);  // solved by f1_if
    if (s >= IC) return;  // the interface table overflowed (status 41)
    const long long sl = (long long)j * IC + s;
    F1Result r;
#pragma unroll
    for (int q = 0; q < NQ; ++q) r.flux[q] = G.ifs[q * IS + sl];
    r.sd_rev = G.ifs[(NQ + 1) * IS + sl];
    const int fl = (int)G.ifs[(NQ + 2) * IS + sl];
    r.have_fwd = (fl & 1) != 0;
    r.have_rev = (fl & 2) != 0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] += r.flux[q];
    sd = fmax(sd, r.sd_rev);
    // the reference's spectral-index local keeps the forward value when the
    // reverse test returns early
    if ((r.have_rev || r.have_fwd) && P_SPEC > ps) ps = P_SPEC;
  };
  // foreign stale contributors, sorted by cell id (= (j, i) order)
  int ns = G.stale_n[t];
  if (ns > KMAX_STALE) ns = KMAX_STALE;
  int sid[KMAX_STALE];
  for (int s = 0; s < ns; ++s) {
    int v = G.stale_id[t * KMAX_STALE + s], p = s;
    while (p > 0 && sid[p - 1] > v) {
      sid[p] = sid[p - 1];
      --p;
    }
    sid[p] = v;
  }
  // ... from tracks below t-1
  for (int s = 0; s < ns; ++s) {
    const long long g0 = sid[s];
    const int j = track_of(G, g0);
    if (j < t - 1) add(j, g0);
  }
  if (t >= 1) {
    const int j = t - 1;
    const int n = G.ntrack[j];
    const long long o = (long long)j * G.cap;
    add(j, o);  // cell 0 (its list may be stale)
    // fresh lists of cells 1..n-2: starts are non-decreasing, so the cells
    // holding gn end at the last start <= gn and form a run downwards
    // last i in [1, n-2] with first_i <= gn, or 0; searched from the end of
    // gn's own list into track t-1 (the cells it overlaps)
    const long long hint = (long long)G.nbr[0 * G.NC + gn] + G.nbr[1 * G.NC + gn] - o;
    const int last = partition_from(1, n - 1, hint, [&](int k) { return G.nbr[2 * G.NC + o + k] <= gn; }) - 1;
    // (list ends are non-decreasing too; empty lists only occur at the start)
    int begin = last;
    while (begin >= 1) {
      const long long g0 = o + begin;
      const int first = G.nbr[2 * G.NC + g0], cnt = G.nbr[3 * G.NC + g0];
      if (cnt > 0 && (long long)first + cnt > gn) --begin;
      else break;
    }
    for (int i = begin + 1; i <= last; ++i) add(j, o + i);
    if (n - 1 > 0) add(j, o + n - 1);  // cell ntrack-1 (stale)
  }
  // ... from track t and above
  for (int s = 0; s < ns; ++s) {
    const long long g0 = sid[s];
    const int j = track_of(G, g0);
    if (j >= t) add(j, g0);
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q) G.f1lo[q * G.NC + gn] = acc[q];
  G.sd[gn] = sd;
  G.pspec[gn] = ps;
}

// ---------------------------------------------------------------------------
// Stage 1 after the fluxes: detectShock and collect_dt's reset (the minimum is
// reduced separately).

GB_HD double collect_cell(const Grid2 &G, int j, int i) {
  if (i >= G.ntrack[j]) return DT_INF;
  const long long g = (long long)j * G.cap + i;
  const double d = G.dtl[g];
  G.dtl[g] = DT_INF;
  G.shocked[g] = G.sd[g] > DETECT_SHOCK_THRESHOLD ? 1 : 0;
  return d;
}

// ---------------------------------------------------------------------------
// Grid::update and the RK3 combines.
//
// iface_move: Interface::move of every interface of the active tracks; at
// stage 1 copyState0 first keeps x0; at stages 2, 3 interfaces iLbnd..iRbnd-1
// then take the combined position (rk3.cpp:121-131, 159-168).  xIm keeps the
// moved position for Cell::update.
GB_HD void iface_move(const Grid2 &G, int j, int i, int stage) {
  const int n = G.ntrack[j];
  if (i > n - 2) return;
  const long long g = (long long)j * G.cap + i;
  if (stage == 1) G.xI0[g] = G.xI[g];
  const int jL = jL_of(G), jR = jR_of(G);
  if (j <= jL || j >= jR) return;
  const double dt = *G.dt;
  double x = G.xI[g];
  x += dt * G.v[g];
  G.xIm[g] = x;
  const int iL = iL_of(G), iR = n - G.ngst;
  if (stage == 2 && i >= iL && i <= iR - 1) x = 3. / 4. * G.xI0[g] + 1. / 4. * x;
  if (stage == 3 && i >= iL && i <= iR - 1) x = 1. / 3. * G.xI0[g] + 2. / 3. * x;
  G.xI[g] = x;
}

// Cell::update (cell.cpp:102-127) of an active cell, the stage's combine and
// cons2prim; at the last stage (3, or 1 with the Euler module) the particle
// injection of every cell (run after evolve by Simu::run).  Every cell copies this stage's grad_f1 into the
// persistent one.
// The starting pressure of cons2prim: the cell's previous pressure (the
// reference's warm start).  With a learned guess (Guess::ON), cons2prim stops
// at a poor warm start (C2PStats::deferred) and those cells search again from
// guess(cons, r, need), the network's pressure; every lane of a warp calls it
// together whether or not its cell is updated, so that it may work across the
// warp, and only when a lane of the warp needs it (Guess::any).  `r` is the
// radius cons2prim divides S_theta by.
struct WarmStart {
  static constexpr bool ON = false;
  GB_HD bool any(bool) const { return false; }
  GB_HD double operator()(const double *, double, bool) const { return 0.; }
};

// cons2prim of one cell at radius r, with its statistics in c2p (calls,
// iterations, fallbacks, max iterations, starts from the learned guess, poor
// warm starts)
template <class Guess>
GB_HD void cell_cons2prim(const Phys &ph, double *cons, double *prim, double r, bool upd, unsigned long long *c2p,
                          const Guess &guess) {
  C2PStats cs;
  if (upd) cons2prim(ph, cons, prim, r, &cs, Guess::ON);
  const int poor = upd ? cs.poor : 0;
  if (Guess::ON) {
    const bool need = upd && cs.deferred;
    if (guess.any(need)) {
      const double pg = guess(cons, r, need);
      if (need) {
        if (isfinite(pg) && pg > 0.) prim[PPP] = pg;  // else the warm start stays
        cons2prim<true>(ph, cons, prim, r, &cs);
        c2p[4] += 1;
      }
    }
  }
  if (upd) {
    c2p[0] += 1;
    c2p[1] += cs.iters;
    c2p[2] += cs.fallback;
    if ((unsigned long long)cs.iters > c2p[3]) c2p[3] = cs.iters;
    c2p[5] += poor;
  }
}

// `live` = false: a lane without a cell (the learned guess' warp-uniform loop).
template <class Guess>
GB_HD void update_cell(const Phys &ph, const Params2 &P, const Grid2 &G, int j, int i, int stage,
                       unsigned long long *c2p, bool live, const Guess &guess) {
  const int n = live ? G.ntrack[j] : 0;
  live = live && i < n;
  const long long g = (long long)j * G.cap + i;
  const int jL = jL_of(G), jR = jR_of(G);
  const int iL = iL_of(G), iR = n - G.ngst;
  const bool active_track = j > jL && j < jR;
  const bool upd = live && active_track && i >= iL + 1 && i <= iR - 1;
  double prim[NQ], cons[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) prim[q] = cons[q] = 0.;
  if (live) load_prim(G, g, prim);
  double dt = 0., r1 = 1., r2 = 1., xn = 0., dxn = 0., dV1 = 0.;
  TrackGeo tj{};
  if (upd) {
    dt = *G.dt;
    const Geom G0 = cell_geom(G, j, g);
    prim2cons(ph, prim, cons, G0.r);
    if (stage == 1) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) G.cons0[q * G.NC + g] = cons[q];
      G.dV0[g] = G0.dV;
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) cons[q] *= G0.dV;
#pragma unroll
    for (int q = 0; q < NQ; ++q) cons[q] += (G.flx[q * G.NC + g - 1] - G.flx[q * G.NC + g]) * dt;
#pragma unroll
    for (int q = 0; q < NQ; ++q) cons[q] += (G.f1lo[q * G.NC + g] - G.f1hi[q * G.NC + g]) * dt;
    tj = tgeo(G, j);
    source_terms(ph, prim, G0, tj, dt, cons);
    {  // Cell::radiativeSourceTerms
      const SynchConst sc{P.Nalpha, P.Nmp, P.Nme};
      const double dg = radiative_source<Cfg2>(ph, sc, prim, G0.dV, dt);
      cons[GMX] += dg;
      cons[GMN] += dg;
    }
    const double xL = G.xIm[g - 1], xR = G.xIm[g];
    const Geom G1 = make_geom((xR + xL) / 2., (xR - xL), tj);
#pragma unroll
    for (int q = 0; q < NQ; ++q) cons[q] = q <= TAU ? cons[q] / G1.dV : qdiv(cons[q], G1.dV);
    r1 = G1.cen_r;
    dV1 = G1.dV;
    xn = G1.r;
    dxn = G1.dr;
  }
  cell_cons2prim(ph, cons, prim, r1, upd, c2p, guess);
  if (stage > 1) {
    if (upd) {
      const double w0 = stage == 2 ? 3. / 4. : 1. / 3.;
      const double w1 = stage == 2 ? 1. / 4. : 2. / 3.;
#pragma unroll
      for (int q = 0; q < NQ; ++q) cons[q] = w0 * G.cons0[q * G.NC + g] * G.dV0[g] + w1 * cons[q] * dV1;
      const double cL = G.xI[g - 1], cR = G.xI[g];  // combined positions
      const Geom G2 = make_geom((cR + cL) / 2., (cR - cL), tj);
#pragma unroll
      for (int q = 0; q < NQ; ++q) cons[q] = q <= TAU ? cons[q] / G2.dV : qdiv(cons[q], G2.dV);
      r2 = G2.r;
      xn = G2.r;
      dxn = G2.dr;
    }
    cell_cons2prim(ph, cons, prim, r2, upd, c2p, guess);
  }
  if (!live) return;
  if (upd) {
    G.x[g] = xn;
    G.dx[g] = dxn;
  } else if (active_track && stage > 1 && i >= 1 && i <= n - 2) {
    // CellGeomFromInterfacePos also moves the ghost cells 1 and ntrack-2
    const double cL = G.xI[g - 1], cR = G.xI[g];
    G.x[g] = (cR + cL) / 2.;
    G.dx[g] = (cR - cL);
  }
  const bool last = stage == (ph.euler ? 1 : 3);  // Grid::evolve ends (rk3.cpp, euler.cpp)
  if (last) {
    const SynchConst sc{P.Nalpha, P.Nmp, P.Nme};
    inject_particles(ph, sc, prim, G.shocked[g] != 0, G.pspec[g]);
  }
  if (active_track || last) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) G.prim[q * G.NC + g] = prim[q];
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q) G.gf1[q * G.NC + g] = G.gf1n[q * G.NC + g];
}

// ---------------------------------------------------------------------------
// Regrid of one active track (Grid::regrid body, 2d.cpp:609-832, with the
// checkCellForRegrid of BM.cpp:246-278), one thread.  The reference walks the
// active cells with a live right bound and edits the track in place; here the
// same walk streams the new track into the scratch rows and copies it back.
// A cell is the reference's whole Cell record: state, geometry, dt_loc, the
// two gradients and the neighbour lists move with it.

struct Rec {
  double prim[NQ], gmv[NQ], gf1[NQ];
  double x, dx, dtl;
  int nbr[4];
  double rifx;  // position of the right interface
};

GB_HD void rec_load(const Grid2 &G, long long g, bool has_rif, Rec &c) {
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    c.prim[q] = G.prim[q * G.NC + g];
    c.gmv[q] = G.gmv[q * G.NC + g];
    c.gf1[q] = G.gf1[q * G.NC + g];
  }
  c.x = G.x[g];
  c.dx = G.dx[g];
  c.dtl = G.dtl[g];
#pragma unroll
  for (int k = 0; k < 4; ++k) c.nbr[k] = G.nbr[k * G.NC + g];
  c.rifx = has_rif ? G.xI[g] : 0.;
}

GB_HD void rec_store(const Grid2 &G, long long g, const Rec &c) {
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    G.rprim[q * G.NC + g] = c.prim[q];
    G.rgmv[q * G.NC + g] = c.gmv[q];
    G.rgf1[q * G.NC + g] = c.gf1[q];
  }
  G.rx[g] = c.x;
  G.rdx[g] = c.dx;
  G.rdtl[g] = c.dtl;
#pragma unroll
  for (int k = 0; k < 4; ++k) G.rnbr[k * G.NC + g] = c.nbr[k];
  G.rxI[g] = c.rifx;
}

struct Target {
  double rmin, rmax;
  int nact;
};

GB_HD int regrid_decision(const Params2 &P, const Rec &c, double target_dr) {
  double dr = c.dx;
  double split_DR = P.split_DR, merge_DR = P.merge_DR;
  if (lfac(c.prim) < 2.) {
    split_DR = P.split_DR_slow;
    merge_DR = P.merge_DR_slow;
  }
  if (dr > split_DR * target_dr) return SPLIT;
  if (dr < merge_DR * target_dr) return MERGE;
  return SKIP;
}

// `live`: the track is the one the criterion measures itself against (its
// bounds and active count change as it is regridded); otherwise `fixed`.
GB_HD void regrid_track(const Phys &ph, const Params2 &P, const Grid2 &G, int j, bool live, Target fixed,
                        unsigned long long *nsplit, unsigned long long *nmerge, unsigned long long *c2p) {
  const int ng = G.ngst, iL = ng - 1;
  const int n0 = G.ntrack[j];
  const long long o = (long long)j * G.cap;
  const TrackGeo tj = tgeo(G, j);
  int ntrack = n0, iR = n0 - ng;
  int out = 0;     // output position of the next emitted cell
  bool changed = false;
  Rec prev, cur, nxt;
  auto emit = [&](const Rec &c) {
    rec_store(G, o + out, c);
    ++out;
  };
  for (int k = 0; k < iL; ++k) {
    Rec c;
    rec_load(G, o + k, true, c);
    emit(c);
  }
  rec_load(G, o + iL, true, prev);
  rec_load(G, o + iL + 1, iL + 1 <= n0 - 2, cur);
  int k = iL + 2;  // next original cell (position i+1)
  int i = iL + 1;
  // current x at position pos (for the live bounds)
  auto x_at = [&](int pos) -> double {
    if (pos < out) return G.rx[o + pos];
    if (pos == i - 1) return prev.x;
    if (pos == i) return cur.x;
    return G.x[o + k + (pos - i - 1)];
  };
  while (i <= iR - 1) {
    Target T = fixed;
    if (live) {
      T.rmin = x_at(iL + 1);
      T.rmax = x_at(iR - 1);
      T.nact = ntrack - 2 * ng;
    }
    const double target_dr = (T.rmax - T.rmin) / T.nact;
    const int action = regrid_decision(P, cur, target_dr);
    if (action == SPLIT && ntrack < G.cap - 1) {
      rec_load(G, o + k, k <= n0 - 2, nxt);
      // Grid::split (2d.cpp:685-764)
      double gC[NQ];
      const double cenL = cen_r(prev.x, prev.dx), cenC = cen_r(cur.x, cur.dx), cenR = cen_r(nxt.x, nxt.dx);
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const double gL = (cur.prim[q] - prev.prim[q]) / (cenC - cenL);
        const double gR = (nxt.prim[q] - cur.prim[q]) / (cenR - cenC);
        gC[q] = minmod(gL, gR);
      }
      const double x_old = cur.x, dl_old = cur.dx;
      Rec A = cur, B = nxt;  // the right half reuses the record of the old right neighbour
      A.x = x_old - dl_old / 4.;
      B.x = x_old + dl_old / 4.;
      A.dx = dl_old / 2.;
      B.dx = dl_old / 2.;
      const double xL = cen_r(A.x, A.dx), xR = cen_r(B.x, B.dx);
      const double xI = A.x + A.dx / 2.;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const double Sc = cur.prim[q];
        A.prim[q] = Sc + gC[q] * (xL - xI);
        B.prim[q] = Sc + gC[q] * (xR - xI);
      }
      A.rifx = x_old;
      B.rifx = cur.rifx;
      emit(prev);
      prev = A;
      cur = B;
      ++ntrack;
      ++iR;
      ++i;
      ++*nsplit;
      changed = true;
      continue;
    }
    if (action == MERGE && ntrack > 2 * ng + 2) {
      rec_load(G, o + k, k <= n0 - 2, nxt);
      // Grid::merge (2d.cpp:767-832)
      const bool left = (prev.dx < nxt.dx && i != ng) || i == (ntrack - 2 * ng) + ng - 1;
      const Rec &vic = left ? prev : nxt;
      double cc[NQ], cv[NQ], cons[NQ];
      prim2cons(ph, cur.prim, cc, cur.x);
      prim2cons(ph, vic.prim, cv, vic.x);
      const double dV_loc = make_geom(cur.x, cur.dx, tj).dV;
      const double dV_vic = make_geom(vic.x, vic.dx, tj).dV;
#pragma unroll
      for (int q = 0; q < NQ; ++q) cons[q] = (cc[q] * dV_loc + cv[q] * dV_vic) / (dV_loc + dV_vic);
      Rec M = cur;
      if (left) M.x = ((vic.x - vic.dx / 2.) + (cur.x + cur.dx / 2.)) / 2.;
      else M.x = ((vic.x + vic.dx / 2.) + (cur.x - cur.dx / 2.)) / 2.;
      M.dx = cur.dx + vic.dx;
      C2PStats cs;
      cons2prim(ph, cons, M.prim, M.x, &cs);
      c2p[0] += 1;
      c2p[1] += cs.iters;
      c2p[2] += cs.fallback;
      if ((unsigned long long)cs.iters > c2p[3]) c2p[3] = cs.iters;
      if (left) {
        M.rifx = cur.rifx;
        emit(M);
        prev = nxt;
      } else {
        M.rifx = nxt.rifx;
        emit(prev);
        prev = M;
      }
      rec_load(G, o + k + 1, k + 1 <= n0 - 2, cur);
      k += 2;
      --ntrack;
      --iR;
      ++i;
      ++*nmerge;
      changed = true;
      continue;
    }
    emit(prev);
    prev = cur;
    rec_load(G, o + k, k <= n0 - 2, cur);
    ++k;
    ++i;
  }
  emit(prev);
  emit(cur);
  for (; k < n0; ++k) {
    Rec c;
    rec_load(G, o + k, k <= n0 - 2, c);
    emit(c);
  }
  if (!changed) return;
  G.ntrack[j] = out;
  for (int p = 0; p < out; ++p) {
    const long long gp = o + p;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      G.prim[q * G.NC + gp] = G.rprim[q * G.NC + gp];
      G.gmv[q * G.NC + gp] = G.rgmv[q * G.NC + gp];
      G.gf1[q * G.NC + gp] = G.rgf1[q * G.NC + gp];
    }
    G.x[gp] = G.rx[gp];
    G.dx[gp] = G.rdx[gp];
    G.dtl[gp] = G.rdtl[gp];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) G.nbr[kk * G.NC + gp] = G.rnbr[kk * G.NC + gp];
    if (p <= out - 2) G.xI[gp] = G.rxI[gp];
  }
}

// Whether any active cell of track j would act against target T (the
// per-cell decision in the original context).  A track with no action leaves
// the regrid untouched, and a live track with no action keeps its target.
GB_HD bool regrid_needed(const Params2 &P, const Grid2 &G, int j, const Target &T, int tid, int nth) {
  const int n = G.ntrack[j], iL = iL_of(G), iR = n - G.ngst;
  const long long o = (long long)j * G.cap;
  const double target_dr = (T.rmax - T.rmin) / T.nact;
  bool any = false;
  for (int i = iL + 1 + tid; i <= iR - 1; i += nth) {
    Rec c;
    for (int q = 0; q < NQ; ++q) c.prim[q] = (q == UU1 || q == UU2) ? G.prim[q * G.NC + o + i] : 0.;
    c.dx = G.dx[o + i];
    const int a = regrid_decision(P, c, target_dr);
    if ((a == SPLIT && n < G.cap - 1) || (a == MERGE && n > 2 * G.ngst + 2)) any = true;
  }
  return any;
}

GB_HD Target track_target(const Grid2 &G, int j) {
  const int n = G.ntrack[j];
  const long long o = (long long)j * G.cap;
  Target T;
  T.rmin = G.x[o + iL_of(G) + 1];
  T.rmax = G.x[o + n - G.ngst - 1];
  T.nact = n - 2 * G.ngst;
  return T;
}

#ifdef __CUDACC__
// ---------------------------------------------------------------------------
// The same regrid walk on the GPU, planned by one warp and executed by the
// block.  The plan reads only what the criterion needs (dr, u_r, u_theta) for
// most cells: 32 lanes test the next 32 original cells against the current
// target at once, and the walk jumps to the first that acts (with no action
// in between, neither the target nor any position changes).  Splits and merges
// are done by lane 0 on full records, whose results go to the scratch rows
// as "new" cells.  The new track is a list of segments -- runs of original
// cells or single new cells -- which all threads then expand from the first
// changed position on.  Scratch per track: seg_start / seg_src (2 cap ints
// from j*cap in rnbr rows 0-1 ... ), new cells in the r* rows at j*cap + id.

struct Desc {  // a cell as the planner sees it
  int orig;     // original index, or -1 - id for a new cell
  double x, dx, u1, u2;
};

__device__ __forceinline__ Desc desc_orig(const Grid2 &G, long long o, int m) {
  Desc d;
  d.orig = m;
  d.x = G.x[o + m];
  d.dx = G.dx[o + m];
  d.u1 = G.prim[UU1 * G.NC + o + m];
  d.u2 = G.prim[UU2 * G.NC + o + m];
  return d;
}

__device__ __forceinline__ int decide(const Params2 &P, double dx, double u1, double u2, double target_dr) {
  double u = 0.;
  u += u1 * u1;
  u += u2 * u2;
  u = sqrt(u);
  const double lf = sqrt(1 + u * u);
  double split_DR = P.split_DR, merge_DR = P.merge_DR;
  if (lf < 2.) {
    split_DR = P.split_DR_slow;
    merge_DR = P.merge_DR_slow;
  }
  if (dx > split_DR * target_dr) return SPLIT;
  if (dx < merge_DR * target_dr) return MERGE;
  return SKIP;
}

// full record of a planner cell (original or new)
__device__ void load_rec(const Grid2 &G, long long o, int n0, const Desc &d, Rec &c, int *rif) {
  if (d.orig >= 0) {
    rec_load(G, o + d.orig, d.orig <= n0 - 2, c);
    *rif = d.orig <= n0 - 2 ? d.orig : -1;
  } else {
    const long long g = o + (-1 - d.orig);
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      c.prim[q] = G.rprim[q * G.NC + g];
      c.gmv[q] = G.rgmv[q * G.NC + g];
      c.gf1[q] = G.rgf1[q * G.NC + g];
    }
    c.x = G.rx[g];
    c.dx = G.rdx[g];
    c.dtl = G.rdtl[g];
#pragma unroll
    for (int k = 0; k < 4; ++k) c.nbr[k] = G.rnbr[k * G.NC + g];
    c.rifx = G.rxI[g];
    *rif = (int)G.rdV[g];
  }
}

// store a new cell; returns its descriptor
__device__ Desc store_new(const Grid2 &G, long long o, int id, const Rec &c, int rif) {
  const long long g = o + id;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    G.rprim[q * G.NC + g] = c.prim[q];
    G.rgmv[q * G.NC + g] = c.gmv[q];
    G.rgf1[q * G.NC + g] = c.gf1[q];
  }
  G.rx[g] = c.x;
  G.rdx[g] = c.dx;
  G.rdtl[g] = c.dtl;
#pragma unroll
  for (int k = 0; k < 4; ++k) G.rnbr[k * G.NC + g] = c.nbr[k];
  G.rxI[g] = c.rifx;
  G.rdV[g] = (double)rif;  // right interface: original index, or -1 (position in rxI)
  Desc d;
  d.orig = -1 - id;
  d.x = c.x;
  d.dx = c.dx;
  d.u1 = c.prim[UU1];
  d.u2 = c.prim[UU2];
  return d;
}

struct PlanOut {
  int nnew, nseg, first;
  unsigned long long splits, merges;
  unsigned long long c2p[4];
};

// warp 0 of the block; returns the plan (valid in lane 0)
__device__ PlanOut regrid_plan(const Phys &ph, const Params2 &P, const Grid2 &G, int j, bool live, Target fixed) {
  const int lane = threadIdx.x & 31;
  const int ng = G.ngst, iL = ng - 1;
  const int n0 = G.ntrack[j];
  const long long o = (long long)j * G.cap;
  int *seg_start = G.rseg + 2 * o;
  int *seg_src = seg_start + G.cap;
  const TrackGeo tj = tgeo(G, j);
  PlanOut R{};
  int ntrack = n0, iR = n0 - ng;
  int out = 0, nseg = 0, nid = 0, first = 1 << 30, run_next = -2;
  double x_first = G.x[o + iL + 1];  // current x at position iL+1 (the live bound)
  auto emit_range = [&](int k0, int k1) {  // originals [k0, k1) at out..
    if (k1 <= k0) return;
    if (!(nseg > 0 && run_next == k0)) {
      if (lane == 0) {
        seg_start[nseg] = out;
        seg_src[nseg] = k0;
      }
      ++nseg;
    }
    if (out != k0 && out < first) first = out;
    if (out <= iL + 1 && out + (k1 - k0) > iL + 1) x_first = G.x[o + k0 + (iL + 1 - out)];
    out += k1 - k0;
    run_next = k1;
  };
  auto emit = [&](const Desc &d) {
    if (d.orig >= 0) {
      emit_range(d.orig, d.orig + 1);
      return;
    }
    if (lane == 0) {
      seg_start[nseg] = out;
      seg_src[nseg] = d.orig;
    }
    ++nseg;
    run_next = -2;
    if (out < first) first = out;
    if (out == iL + 1) x_first = d.x;
    ++out;
  };
  emit_range(0, iL);
  Desc prev = desc_orig(G, o, iL), cur = desc_orig(G, o, iL + 1);
  int k = iL + 2;
  int i = iL + 1;
  while (i <= iR - 1) {
    Target T = fixed;
    if (live) {
      T.rmin = (iL + 1 == i - 1) ? prev.x : ((iL + 1 == i) ? cur.x : x_first);
      const int pr = iR - 1;
      T.rmax = (pr == i) ? cur.x : ((pr == i - 1) ? prev.x : G.x[o + k + (pr - i - 1)]);
      T.nact = ntrack - 2 * ng;
    }
    const double target_dr = (T.rmax - T.rmin) / T.nact;
    int act;
    if (cur.orig >= 0) {
      // lanes test originals cur.orig + lane at positions i + lane
      const int m = cur.orig + lane;
      const bool valid = i + lane <= iR - 1;
      int a = SKIP;
      if (valid) a = decide(P, G.dx[o + m], G.prim[UU1 * G.NC + o + m], G.prim[UU2 * G.NC + o + m], target_dr);
      const bool acts = valid && ((a == SPLIT && ntrack < G.cap - 1) || (a == MERGE && ntrack > 2 * ng + 2));
      const unsigned ball = __ballot_sync(0xffffffffu, acts);
      const unsigned vball = __ballot_sync(0xffffffffu, valid);
      const int f = ball ? __ffs(ball) - 1 : __popc(vball);
      if (f > 0) {  // f no-op cells at positions i .. i+f-1
        emit(prev);
        emit_range(cur.orig, cur.orig + f - 1);
        const int c0 = cur.orig;
        prev = desc_orig(G, o, c0 + f - 1);
        cur = desc_orig(G, o, c0 + f);
        k = c0 + f + 1;
        i += f;
        continue;
      }
      act = __shfl_sync(0xffffffffu, a, 0);
    } else {
      act = decide(P, cur.dx, cur.u1, cur.u2, target_dr);
      if (!((act == SPLIT && ntrack < G.cap - 1) || (act == MERGE && ntrack > 2 * ng + 2))) act = SKIP;
    }
    if (act == SPLIT) {
      // Grid::split (2d.cpp:685-764), by lane 0
      Desc dA, dB;
      if (lane == 0) {
        Rec L, C, N;
        int rL, rC, rN;
        load_rec(G, o, n0, prev, L, &rL);
        load_rec(G, o, n0, cur, C, &rC);
        load_rec(G, o, n0, desc_orig(G, o, k), N, &rN);
        double gC[NQ];
        const double cenL = cen_r(L.x, L.dx), cenC = cen_r(C.x, C.dx), cenR = cen_r(N.x, N.dx);
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          const double gL = (C.prim[q] - L.prim[q]) / (cenC - cenL);
          const double gR = (N.prim[q] - C.prim[q]) / (cenR - cenC);
          gC[q] = minmod(gL, gR);
        }
        const double x_old = C.x, dl_old = C.dx;
        Rec A = C, B = N;
        A.x = x_old - dl_old / 4.;
        B.x = x_old + dl_old / 4.;
        A.dx = dl_old / 2.;
        B.dx = dl_old / 2.;
        const double xL = cen_r(A.x, A.dx), xR = cen_r(B.x, B.dx);
        const double xI = A.x + A.dx / 2.;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          const double Sc = C.prim[q];
          A.prim[q] = Sc + gC[q] * (xL - xI);
          B.prim[q] = Sc + gC[q] * (xR - xI);
        }
        A.rifx = x_old;
        B.rifx = C.rifx;
        dA = store_new(G, o, nid, A, -1);
        dB = store_new(G, o, nid + 1, B, rC);
      }
      nid += 2;
      emit(prev);
      prev.orig = __shfl_sync(0xffffffffu, dA.orig, 0);
      prev.x = __shfl_sync(0xffffffffu, dA.x, 0);
      prev.dx = __shfl_sync(0xffffffffu, dA.dx, 0);
      prev.u1 = __shfl_sync(0xffffffffu, dA.u1, 0);
      prev.u2 = __shfl_sync(0xffffffffu, dA.u2, 0);
      cur.orig = __shfl_sync(0xffffffffu, dB.orig, 0);
      cur.x = __shfl_sync(0xffffffffu, dB.x, 0);
      cur.dx = __shfl_sync(0xffffffffu, dB.dx, 0);
      cur.u1 = __shfl_sync(0xffffffffu, dB.u1, 0);
      cur.u2 = __shfl_sync(0xffffffffu, dB.u2, 0);
      ++ntrack;
      ++iR;
      ++i;
      ++R.splits;
      continue;
    }
    if (act == MERGE) {
      // Grid::merge (2d.cpp:767-832), by lane 0
      const Desc nxt = desc_orig(G, o, k);
      const bool left = (prev.dx < nxt.dx && i != ng) || i == (ntrack - 2 * ng) + ng - 1;
      Desc dM;
      if (lane == 0) {
        Rec C, V;
        int rC, rV;
        load_rec(G, o, n0, cur, C, &rC);
        load_rec(G, o, n0, left ? prev : nxt, V, &rV);
        double cc[NQ], cv[NQ], cons[NQ];
        prim2cons(ph, C.prim, cc, C.x);
        prim2cons(ph, V.prim, cv, V.x);
        const double dV_loc = make_geom(C.x, C.dx, tj).dV;
        const double dV_vic = make_geom(V.x, V.dx, tj).dV;
#pragma unroll
        for (int q = 0; q < NQ; ++q) cons[q] = (cc[q] * dV_loc + cv[q] * dV_vic) / (dV_loc + dV_vic);
        Rec M = C;
        if (left) M.x = ((V.x - V.dx / 2.) + (C.x + C.dx / 2.)) / 2.;
        else M.x = ((V.x + V.dx / 2.) + (C.x - C.dx / 2.)) / 2.;
        M.dx = C.dx + V.dx;
        C2PStats cs;
        cons2prim(ph, cons, M.prim, M.x, &cs);
        R.c2p[0] += 1;
        R.c2p[1] += cs.iters;
        R.c2p[2] += cs.fallback;
        if ((unsigned long long)cs.iters > R.c2p[3]) R.c2p[3] = cs.iters;
        int rM;
        if (left) {
          M.rifx = C.rifx;
          rM = rC;
        } else {
          M.rifx = V.rifx;
          rM = rV;
        }
        dM = store_new(G, o, nid, M, rM);
      }
      nid += 1;
      dM.orig = __shfl_sync(0xffffffffu, dM.orig, 0);
      dM.x = __shfl_sync(0xffffffffu, dM.x, 0);
      dM.dx = __shfl_sync(0xffffffffu, dM.dx, 0);
      dM.u1 = __shfl_sync(0xffffffffu, dM.u1, 0);
      dM.u2 = __shfl_sync(0xffffffffu, dM.u2, 0);
      if (left) {
        emit(dM);
        prev = nxt;
      } else {
        emit(prev);
        prev = dM;
      }
      cur = desc_orig(G, o, k + 1);
      k += 2;
      --ntrack;
      --iR;
      ++i;
      ++R.merges;
      continue;
    }
    emit(prev);
    prev = cur;
    cur = desc_orig(G, o, k);
    ++k;
    ++i;
  }
  emit(prev);
  emit(cur);
  emit_range(k, n0);
  R.nnew = out;
  R.nseg = nseg;
  R.first = first;
  return R;
}

// all threads of the block: expand the plan from the first changed position
__device__ void regrid_execute(const Grid2 &G, int j, int n0, int nnew, int nseg, int first) {
  const long long o = (long long)j * G.cap;
  const int *seg_start = G.rseg + 2 * o;
  const int *seg_src = seg_start + G.cap;
  if (first >= nnew && nnew == n0) return;
  // stage the new track from `first` in the rows of a second scratch (the
  // gf1n rows: overwritten by the next transverse-gradient pass anyway) ...
  // positions >= first are written to t*, then copied back
  double *tp = G.gf1n;  // [NQ][NC]: prim
  double *tgm = G.cons0;  // [NQ][NC]: grad_mv
  double *tgf = G.f1lo;   // [NQ][NC]: grad_f1
  double *tx = G.xI0, *tdx = G.xIm, *tdtl = G.v, *txI = G.lL;
  int *tnb = G.rnbr2;     // [4][NC]
  for (int p = first + threadIdx.x; p < nnew; p += blockDim.x) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (seg_start[mid] <= p) lo = mid;
      else hi = mid - 1;
    }
    const int src = seg_src[lo];
    const long long gp = o + p;
    if (src >= 0) {
      const long long gk = o + src + (p - seg_start[lo]);
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        tp[q * G.NC + gp] = G.prim[q * G.NC + gk];
        tgm[q * G.NC + gp] = G.gmv[q * G.NC + gk];
        tgf[q * G.NC + gp] = G.gf1[q * G.NC + gk];
      }
      tx[gp] = G.x[gk];
      tdx[gp] = G.dx[gk];
      tdtl[gp] = G.dtl[gk];
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) tnb[kk * G.NC + gp] = G.nbr[kk * G.NC + gk];
      txI[gp] = G.xI[gk];
    } else {
      const long long gn = o + (-1 - src);
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        tp[q * G.NC + gp] = G.rprim[q * G.NC + gn];
        tgm[q * G.NC + gp] = G.rgmv[q * G.NC + gn];
        tgf[q * G.NC + gp] = G.rgf1[q * G.NC + gn];
      }
      tx[gp] = G.rx[gn];
      tdx[gp] = G.rdx[gn];
      tdtl[gp] = G.rdtl[gn];
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) tnb[kk * G.NC + gp] = G.rnbr[kk * G.NC + gn];
      const int rif = (int)G.rdV[gn];
      txI[gp] = rif >= 0 ? G.xI[o + rif] : G.rxI[gn];
    }
  }
  __syncthreads();
  for (int p = first + threadIdx.x; p < nnew; p += blockDim.x) {
    const long long gp = o + p;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      G.prim[q * G.NC + gp] = tp[q * G.NC + gp];
      G.gmv[q * G.NC + gp] = tgm[q * G.NC + gp];
      G.gf1[q * G.NC + gp] = tgf[q * G.NC + gp];
    }
    G.x[gp] = tx[gp];
    G.dx[gp] = tdx[gp];
    G.dtl[gp] = tdtl[gp];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) G.nbr[kk * G.NC + gp] = tnb[kk * G.NC + gp];
    if (p <= nnew - 2) G.xI[gp] = txI[gp];
  }
  __syncthreads();
  if (threadIdx.x == 0) G.ntrack[j] = nnew;
}
#endif  // __CUDACC__

}  // namespace d2
}  // namespace gb
