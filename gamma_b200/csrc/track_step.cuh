// One CTA advances one run (one 1D track of cells) through whole RK3 steps.
//
// Per step (src/simu.cpp:79-105): [regrid] -> reset shocks -> ghosts ->
// stage-1 CFL candidates -> per-run dt (block min) -> stage-1 update ->
// ghosts -> stage-2 fluxes+update+RK combine -> ghosts -> stage-3 -> inject.
// With the Euler module (Timestep/euler.cpp:12-19) the step ends after the
// stage-1 update: inject, and no RK combine.
//
// Each stage is one left-to-right sweep over the track in chunks of BS cells
// (one interface and one cell per thread).  A chunk stages the stencil
// (cells a-1 .. a+BS+1) in shared memory, computes the BS interfaces
// a .. a+BS-1 (PLM + HLLC at the contact-speed interface), then updates cells
// a .. a+BS-1 in place.  The old state of cell a+BS-1 and the results of
// interface a+BS-1 are carried to the next chunk, so the in-place update never
// feeds a neighbour's stencil.  Runs are independent (own dt, own regrid), so
// a CTA takes runs from a work queue and can advance each by many steps
// without any grid-wide synchronisation.
#pragma once

#include "gamma_problem.h"
#include "mlp.cuh"
#include "physics.cuh"
#include "regrid.cuh"

#ifdef GB_SWEEP_NOINLINE
#define GB_SWEEP_ATTR __noinline__
#else
#define GB_SWEEP_ATTR __forceinline__
#endif

namespace gb {

// Device view of the pooled structure-of-arrays state.  Run r owns cells
// [off[r], off[r]+cap[r]) of every per-cell array.  Primitive slot q is stored
// at row (q < 3 ? q : q-1): slot 3 is identically zero in 1D.
struct Tracks {
  double *prim;     // [NQS][N]
  double *x, *dx;   // cell centre and width at step start
  double *dtl;      // Cell::dt_loc, carried between steps
  double *xI;       // interface i sits between cells i and i+1
  double *u0;       // [NQS][N] step-start cons * dV (stage combine)
  double *xI0;      // step-start interface positions
  double *fl1;      // [NQS][N] stage-1 interface fluxes (kept from the CFL pass)
  double *v1;       // stage-1 interface velocities
  double *sd, *pspec;
  uint8_t *shocked;
  long long N;      // row stride
  const long long *off;
  const int *cap;
  RunState *run;    // per-run scalars (ntrack, t, dt, it, status)
  const double *par;  // [nruns][gamma_problem::PARAM_WORDS] problem parameters
  RegridScratch rg;
  const float *mlp;  // learned cons2prim guess parameters (kernels built with GUESS only)
};

template <class Cfg>
struct Slots {
  static constexpr int NQS = Cfg::NQ - 1;
  __device__ __forceinline__ static constexpr int q_of(int s) { return s < 3 ? s : s + 1; }
};

struct StepStats {
  unsigned long long c2p_calls;
  unsigned long long c2p_iters;
  unsigned long long c2p_fallbacks;
  unsigned long long zone_updates;
  unsigned long long splits, merges;
  int c2p_max_iters;
  int status;
  unsigned long long c2p_guesses;  // cons2prim calls started from the learned guess
  unsigned long long c2p_poor;     // cons2prim calls whose warm start was poor (c2p_warm_start_poor)
  unsigned long long learned;      // launches of the step with the learned guess that ran
};


// BS threads advance one run; each sweep chunk holds CPT cells per thread
// (CH = BS * CPT), which a thread takes in turn.  Hooks: the problem module
// (include/gamma_problem.h), whose hooks run where the reference calls its
// own: userBoundaries in ghosts, userKinematics and userSourceTerms in the
// sweep, cons2prim_user in cons2prim, checkCellForRegrid in regrid_track.
template <class Cfg, class Hooks, int BS, bool GUESS = false, int CPT = 1>
struct TrackStep {
  static constexpr int NQ = Cfg::NQ;
  static constexpr int NQS = Cfg::NQ - 1;
  static constexpr int CH = BS * CPT;  // cells and interfaces per chunk
  static constexpr int NC = CH + 3;    // staged cells per chunk: a-1 .. a+CH+1

  struct Smem {
    double cp[NQS][NC];  // staged primitives
    double cx[NC], cdx[NC], cen[NC];
    double fl[NQS][CH + 1];  // interface fluxes; slot 0 = carry (interface a-1)
    double lL[CH + 1], lR[CH + 1], v[CH + 1];
    double xold[CH + 1], xnew[CH + 1], xcmb[CH + 1];
    double gp[NQS][NC];  // gradient between slots k and k+1 (grad())
    double red[BS / 32];
    double edge[4];  // x, dx of the left and right edge cells this stage
    int ints[4];
  };

  // --- helpers ------------------------------------------------------------

  __device__ static double block_min(Smem &sm, double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sm.red[w] = v;
    __syncthreads();
    double r = sm.red[0];
#pragma unroll
    for (int k = 1; k < BS / 32; ++k) r = fmin(r, sm.red[k]);
    __syncthreads();
    return r;
  }

  __device__ static void load_prim(const Tracks &T, long long g, double *p) {
#pragma unroll
    for (int s = 0; s < NQS; ++s) p[Slots<Cfg>::q_of(s)] = T.prim[s * T.N + g];
    p[UU2] = 0.;
  }
  __device__ static void store_prim(const Tracks &T, long long g, const double *p) {
#pragma unroll
    for (int s = 0; s < NQS; ++s) T.prim[s * T.N + g] = p[Slots<Cfg>::q_of(s)];
  }

  // Ghost cells and ghost interfaces (Grid::updateGhosts, 1d.cpp:217-246) and
  // the problem's boundary hook.  edge: geometry of the two edge cells.
  __device__ static void ghosts(const Tracks &T, const Phys &ph, const gamma_problem::HookArgs &A, long long off,
                                int n, const double *edge) {
    const int ng = ph.ngst, iL = ng - 1, iR = n - ng;
    const int tid = threadIdx.x;
    if (tid < 2 * ng) {
      const bool left = tid < ng;
      const int e = left ? iL + 1 : iR - 1;
      const int i = left ? tid : iR + (tid - ng);
      const long long ge = off + e, gi = off + i;
      double p[NQ];
      load_prim(T, ge, p);
      // the ghost's centre as updateGhosts shifts it (1d.cpp:221, 234)
      const double gx = left ? edge[0] - (iL - i + 1) * edge[1] : edge[2] + (i - iR + 1) * edge[3];
      Hooks::user_boundaries(A, i, gx, p);  // Grid::userBoundaries (1d.cpp:244)
      store_prim(T, gi, p);
      T.dtl[gi] = T.dtl[ge];
      if (Cfg::SHOCK) {
        T.sd[gi] = T.sd[ge];
        T.pspec[gi] = T.pspec[ge];
        T.shocked[gi] = T.shocked[ge];
      }
    }
    // ghost interfaces: left 0..iL-1 from iL+1; right iR..n-2 from iR-1
    if (tid >= 32 && tid < 32 + ng) {
      const int i = tid - 32;
      if (i <= iL - 1) T.xI[off + i] = T.xI[off + iL + 1] - (iL - i + 1) * edge[1];
      const int j = iR + i;
      if (j <= n - 2) T.xI[off + j] = T.xI[off + iR - 1] + (j - iR) * edge[3];
    }
  }

  // Geometry of cell i during the current stage.  Active cells: the step-start
  // arrays (stage 1) or the span of their interfaces (stages 2, 3: set by
  // Cell::move and CellGeomFromInterfacePos).  Ghosts: shifted copies of the
  // edge cells (updateGhosts).
  __device__ static void cell_geom(const Tracks &T, const Smem &sm, long long off, int n, int ng, int stage,
                                   int i, const double *xIold_prev, double *gx, double *gdx) {
    const int iL = ng - 1, iR = n - ng;
    if (i <= iL) {
      *gx = sm.edge[0] - (iL - i + 1) * sm.edge[1];
      *gdx = sm.edge[1];
    } else if (i >= iR) {
      *gx = sm.edge[2] + (i - iR + 1) * sm.edge[3];
      *gdx = sm.edge[3];
    } else if (stage == 1) {
      *gx = T.x[off + i];
      *gdx = T.dx[off + i];
    } else {
      const double xL = xIold_prev ? *xIold_prev : T.xI[off + i - 1];
      const double xR = T.xI[off + i];
      *gx = (xR + xL) / 2.;
      *gdx = (xR - xL);
    }
  }

  // Reconstructed left/right states at interface i from staged cells
  // (Grid::reconstructStates, 1d.cpp:370-461).  c = slot of cell i.
  __device__ static void reconstruct(const Smem &sm, const Phys &ph, int i, int n, int c, double xI,
                                     FState<Cfg> &L, FState<Cfg> &R) {
    if (i == 0 || i == n - 2) {
#pragma unroll
      for (int s = 0; s < NQS; ++s) {
        L.prim[Slots<Cfg>::q_of(s)] = sm.cp[s][c];
        R.prim[Slots<Cfg>::q_of(s)] = sm.cp[s][c + 1];
      }
    } else {
      // cells i-1 .. i+2 (i+2 <= n-1 for every interior interface)
      const double cenL = sm.cen[c], cenR = sm.cen[c + 1];
      const double dL = xI - cenL, dR = xI - cenR;
#pragma unroll
      for (int s = 0; s < NQS; ++s) {
        const double qL = sm.cp[s][c], qR = sm.cp[s][c + 1];
        // grad() of 1d.cpp:262-274, formed once per cell pair in the sweep
        const double gN = sm.gp[s][c];
        double gL = sm.gp[s][c - 1];
        double gR = sm.gp[s][c + 1];
        gL = minmod(gL, gN);
        gR = minmod(gR, gN);
        L.prim[Slots<Cfg>::q_of(s)] = qL + gL * dL;
        R.prim[Slots<Cfg>::q_of(s)] = qR + gR * dR;
      }
    }
    L.prim[UU2] = 0.;
    R.prim[UU2] = 0.;
    fill_state<Cfg>(ph, L);
    fill_state<Cfg>(ph, R);
  }

  // Cell::update_dt, moving direction (cell.cpp:47-74).  Returns false on a
  // negative candidate (the reference's exit(30)).
  __device__ static bool dt_candidate(double a, double lR_left, double v_right, double lL_right, double v_left,
                                      double *cand) {
    double dL = (lR_left > v_right) ? a / (lR_left - v_right) : DT_INF;
    double dR = (lL_right < v_left) ? a / (v_left - lL_right) : DT_INF;
    *cand = fmin(dL, dR);
    return !(*cand < 0);
  }

  __device__ static void count_c2p(StepStats &st, const C2PStats &cs, int poor) {
    st.c2p_calls++;
    st.c2p_poor += poor;
    st.c2p_iters += cs.iters;
    st.c2p_fallbacks += cs.fallback;
    st.c2p_max_iters = max(st.c2p_max_iters, cs.iters);
  }

  // cons2prim of one cell, with the learned guess (GUESS): the search stops at
  // a poor warm start (C2PStats::deferred) and those cells search again from
  // the network's pressure (a non-finite or non-positive guess keeps the warm
  // one).  Every lane of the warp calls (upd = false: no cell); the network
  // runs only when a lane of the warp needs it, and the second search is the
  // out-of-line copy, so that the step's own loop stays as without the guess.
  __device__ static void cell_cons2prim(const mlp::InferSmem *inf, const Phys &ph, double *cons, double *prim,
                                        bool upd, StepStats &st, const double *par) {
    C2PStats cs;
    if (upd) cons2prim<Cfg, Hooks>(ph, cons, prim, &cs, par, GUESS);
    const int poor = upd ? cs.poor : 0;
    if (GUESS) {
      const bool need = upd && cs.deferred;
      if (__any_sync(0xffffffffu, need)) {
        const double pg = mlp::warp_guess_pressure(*inf, cons[DEN], cons[TAU], cons[SS1], need);
        if (need) {
          if (isfinite(pg) && pg > 0.) prim[PPP] = pg;
          cons2prim<Cfg, Hooks, true>(ph, cons, prim, &cs, par);
          st.c2p_guesses++;
        }
      }
    }
    if (upd) count_c2p(st, cs, poor);
  }

  // --- one stage sweep ------------------------------------------------------
  // mode 0: stage-1 CFL candidates only (returns the run's min dt_loc and
  //         resets dt_loc); mode 1: fluxes + update (+ RK combine for stage>1).
  // Inlined into the step (measured faster than one shared out-of-line copy,
  // whose call frame costs local-memory traffic).
  __device__ GB_SWEEP_ATTR static double sweep(const Tracks &T, const Phys &ph, const gamma_problem::HookArgs &A,
                                              const SynchConst &sc,
                                 Smem &sm, long long off, int n, int stage, int mode, double dt, double t,
                                 StepStats &st, const mlp::InferSmem *inf) {
    const int tid = threadIdx.x;
    const int ng = ph.ngst, iL = ng - 1, iR = n - ng;
    const double w0 = stage == 2 ? 3. / 4. : 1. / 3.;
    const double w1 = stage == 2 ? 1. / 4. : 2. / 3.;
    double run_min = DT_INF;

    for (int a = 0; a < n; a += CH) {
      // ---- stage cells a-1 .. a+CH+1 (slot k <-> cell a-1+k); slot 0 is carried
      for (int k = tid + 1; k < NC; k += BS) {
        const int i = a - 1 + k;
        if (i < n) {
          const long long g = off + i;
#pragma unroll
          for (int s = 0; s < NQS; ++s) sm.cp[s][k] = T.prim[s * T.N + g];
          double gx, gdx;
          // cell a's left interface was rewritten by the previous chunk: use its carried old position
          cell_geom(T, sm, off, n, ng, stage, i, (k == 1 && a > 0) ? &sm.xold[0] : nullptr, &gx, &gdx);
          sm.cx[k] = gx;
          sm.cdx[k] = gdx;
          sm.cen[k] = make_geom<Cfg>(gx, gdx).cen;
        }
      }
      __syncthreads();
      if (!(mode == 1 && stage == 1)) {
        // grad() between staged cells k and k+1: (q[k+1] - q[k]) / (cen[k+1] - cen[k]),
        // each used by the three interfaces around it (slots past the track end unused)
        for (int k = tid; k < NC - 1; k += BS) {
          if ((a > 0 || k > 0) && a + k < n) {  // slots k and k+1 both hold cells
            const double d = sm.cen[k + 1] - sm.cen[k];
            // in the reference's order unless every formula may move (FAST_RIEMANN):
            // minmod of two equal slopes is 0 (1d.cpp:250-260), and a split's two
            // halves make such ties on purpose (their pair gradient is the split's)
            if (Cfg::FAST_RIEMANN) {
              const double rd = 1. / d;
#pragma unroll
              for (int s = 0; s < NQS; ++s) sm.gp[s][k] = (sm.cp[s][k + 1] - sm.cp[s][k]) * rd;
            } else {
#pragma unroll
              for (int s = 0; s < NQS; ++s) sm.gp[s][k] = qdiv(sm.cp[s][k + 1] - sm.cp[s][k], d);
            }
          }
        }
        __syncthreads();
      }

      // ---- interfaces i = a + tid + u BS
#pragma unroll 1
      for (int u = 0; u < CPT; ++u) {
      const int tt = tid + u * BS;
      const int i = a + tt;
      const bool has_if = i <= n - 2;
      const int c = tt + 1;  // slot of cell i
      double myflux[NQ];
#pragma unroll
      for (int q = 0; q < NQ; ++q) myflux[q] = 0.;
      double my_lL = 0, my_lR = 0, my_v = 0, my_xold = 0, my_xnew = 0, my_xcmb = 0;
      if (has_if) {
        const long long gi = off + i;
        const double xI = T.xI[gi];
        my_xold = xI;
        if (mode == 1 && stage == 1) {
          // stage-1 fluxes and velocities were solved by the CFL pass
          my_v = T.v1[gi];
#pragma unroll
          for (int s = 0; s < NQS; ++s) myflux[Slots<Cfg>::q_of(s)] = T.fl1[s * T.N + gi];
        } else {
          FState<Cfg> L, R;
          reconstruct(sm, ph, i, n, c, xI, L, R);
          const Waves w = compute_lambda<Cfg>(ph, L, R);
          double v = ph.vi * w.lS;
          Hooks::user_kinematics(A, i, &v);  // Grid::userKinematics (1d.cpp:749)
          my_lL = w.lL;
          my_lR = w.lR;
          my_v = v;
          hllc_flux<Cfg>(L, R, w, v, iface_area<Cfg>(xI), myflux);
          if (Cfg::SHOCK) {  // measureShock into cell i (radiation_sph.cpp:160-175)
            double Sd, ps;
            const bool have = compute_Sd<Cfg>(ph, L, R, &Sd, &ps);
            const double sd0 = fmax(T.sd[gi], Sd);
            T.sd[gi] = sd0;
            if (have && ps > T.pspec[gi]) T.pspec[gi] = ps;
            if (stage == 1) T.shocked[gi] = sd0 > DETECT_SHOCK_THRESHOLD ? 1 : 0;  // detectShock
          }
          if (mode == 0) {  // keep the stage-1 solution for the update pass
            T.v1[gi] = v;
#pragma unroll
            for (int s = 0; s < NQS; ++s) T.fl1[s * T.N + gi] = myflux[Slots<Cfg>::q_of(s)];
          }
        }
        if (mode == 1) {
          // Interface::move, then the RK combine of interface positions
          my_xnew = xI + dt * my_v;
          if (stage == 1) {
            T.xI0[gi] = xI;
            my_xcmb = my_xnew;
          } else if (i >= iL && i <= iR - 1) {
            my_xcmb = w0 * T.xI0[gi] + w1 * my_xnew;
          } else {
            my_xcmb = my_xnew;
          }
          T.xI[gi] = my_xcmb;
        }
      }
      // cell n-1 has no interface of its own; as for every cell, the shock
      // detector result of the last real interface is already in place.
      sm.lL[tt + 1] = my_lL;
      sm.lR[tt + 1] = my_lR;
      sm.v[tt + 1] = my_v;
      if (mode == 1) {
        sm.xold[tt + 1] = my_xold;
        sm.xnew[tt + 1] = my_xnew;
        sm.xcmb[tt + 1] = my_xcmb;
#pragma unroll
        for (int s = 0; s < NQS; ++s) sm.fl[s][tt + 1] = myflux[Slots<Cfg>::q_of(s)];
      }
      }
      __syncthreads();

      // ---- cells i = a + tid + u BS
#pragma unroll 1
      for (int u = 0; u < CPT; ++u) {
      const int tt = tid + u * BS;
      const int i = a + tt;
      const int c = tt + 1;
      if (i < n) {
        const long long g = off + i;
        if (i >= 1 && i <= n - 2 && (mode == 0 || stage > 1)) {
          double cand;
          if (!dt_candidate(sm.cdx[c], sm.lR[tt], sm.v[tt + 1], sm.lL[tt + 1], sm.v[tt], &cand)) {
            st.status = 30;
            cand = DT_INF;
          }
          const double d = fmin(T.dtl[g], cand);
          if (mode == 0) {
            run_min = fmin(run_min, d);
            T.dtl[g] = DT_INF;  // collect_dt resets (1d.cpp:785)
          } else {
            T.dtl[g] = d;
          }
        } else if (mode == 0) {
          run_min = fmin(run_min, T.dtl[g]);
          T.dtl[g] = DT_INF;
        }
      }

      if (mode == 1) {
        // Cell::update (cell.cpp:102-127).  Written as straight-line blocks
        // under `upd` so that, with the learned guess, the whole warp meets at
        // each inference.
        const bool upd = i >= iL + 1 && i <= iR - 1;
        const long long g = off + i;
        double prim[NQ], cons[NQ];
        Geom G1;
        if (upd) {
#pragma unroll
          for (int s = 0; s < NQS; ++s) prim[Slots<Cfg>::q_of(s)] = sm.cp[s][c];
          prim[UU2] = 0.;
          const Geom G0 = make_geom<Cfg>(sm.cx[c], sm.cdx[c]);
          prim2cons<Cfg>(ph, prim, cons);
#pragma unroll
          for (int q = 0; q < NQ; ++q) cons[q] *= G0.dV;
          if (stage == 1) {
#pragma unroll
            for (int s = 0; s < NQS; ++s) T.u0[s * T.N + g] = cons[Slots<Cfg>::q_of(s)];
          }
#pragma unroll
          for (int s = 0; s < NQS; ++s) {
            const int q = Slots<Cfg>::q_of(s);
            cons[q] += (sm.fl[s][tt] - sm.fl[s][tt + 1]) * dt;
          }
          if (Cfg::SPH) {  // Cell::sourceTerms, 1D (rel_sph.cpp:452-466)
            double p = prim[PPP];
            double r = G0.x, dr = G0.dx, dV = G0.dV;
            double r1 = r - dr / 2., r2 = r + dr / 2.;
            double rsq = (r2 * r2 + r1 * r1 + r2 * r1) / 3.;
            cons[SS1] += (2. * p) * (r / rsq) * dV * dt;
          }
          if (Cfg::CYL) {  // Cell::sourceTerms of rel_cyl.cpp:358-364, r = G.x[r_]
            cons[SS1] += prim[PPP] / G0.x * G0.dV * dt;
          }
          Hooks::user_source_terms(A, G0.x, G0.dx, G0.dV, prim, cons, dt);  // Cell::userSourceTerms
          if (Cfg::SYNCH) {
            const double dg = radiative_source<Cfg>(ph, sc, prim, G0.dV, dt);
            cons[GMX] += dg;
            cons[GMN] += dg;
          }
          G1 = geom_between<Cfg>(sm.xnew[tt], sm.xnew[tt + 1]);
          if (Cfg::FAST) {
            const double rdV1 = 1. / G1.dV;
#pragma unroll
            for (int q = 0; q < NQ; ++q) cons[q] *= rdV1;
          } else {
#pragma unroll
            for (int q = 0; q < NQ; ++q) cons[q] = q <= TAU ? cons[q] / G1.dV : qdiv(cons[q], G1.dV);
          }
        }
        // every lane of the warp meets here (the network works across it)
        cell_cons2prim(inf, ph, cons, prim, upd, st, A.par);
        if (stage > 1) {
          if (upd) {  // RK3 combine (rk3.cpp:27-55, 63-92)
#pragma unroll
            for (int s = 0; s < NQS; ++s) {
              const int q = Slots<Cfg>::q_of(s);
              cons[q] = w0 * T.u0[s * T.N + g] + w1 * cons[q] * G1.dV;
            }
            const Geom G2 = geom_between<Cfg>(sm.xcmb[tt], sm.xcmb[tt + 1]);
            if (Cfg::FAST) {
              const double rdV2 = 1. / G2.dV;
#pragma unroll
              for (int q = 0; q < NQ; ++q) cons[q] *= rdV2;
            } else {
#pragma unroll
              for (int q = 0; q < NQ; ++q) cons[q] = q <= TAU ? cons[q] / G2.dV : qdiv(cons[q], G2.dV);
            }
          }
          cell_cons2prim(inf, ph, cons, prim, upd, st, A.par);
        }
        if (upd) {
          if (Cfg::SYNCH && stage == (ph.euler ? 1 : 3)) {  // radiation_injectParticles, active cells
            inject_particles<Cfg>(ph, sc, prim, T.shocked[g] != 0, T.pspec[g]);
          }
          store_prim(T, g, prim);
        }
      }
      }
      __syncthreads();
      // ---- carry cell a+CH-1 and interface a+CH-1 to the next chunk
      if (tid == 0) {
        sm.lL[0] = sm.lL[CH];
        sm.lR[0] = sm.lR[CH];
        sm.v[0] = sm.v[CH];
        sm.xold[0] = sm.xold[CH];
        sm.xnew[0] = sm.xnew[CH];
        sm.xcmb[0] = sm.xcmb[CH];
        sm.cx[0] = sm.cx[CH];
        sm.cdx[0] = sm.cdx[CH];
        sm.cen[0] = sm.cen[CH];
      }
      if (tid < NQS) {
        sm.fl[tid][0] = sm.fl[tid][CH];
        sm.cp[tid][0] = sm.cp[tid][CH];
      }
      __syncthreads();
    }
    return run_min;
  }

  // Edge-cell geometry for the current stage (written to sm.edge)
  __device__ static void edge_geom(const Tracks &T, Smem &sm, long long off, int n, int ng, int stage) {
    if (threadIdx.x == 0) {
      const int e[2] = {ng, n - ng - 1};
      for (int k = 0; k < 2; ++k) {
        const long long g = off + e[k];
        double gx, gdx;
        if (stage == 1) {
          gx = T.x[g];
          gdx = T.dx[g];
        } else {
          const double xL = T.xI[g - 1], xR = T.xI[g];
          gx = (xR + xL) / 2.;
          gdx = (xR - xL);
        }
        sm.edge[2 * k] = gx;
        sm.edge[2 * k + 1] = gdx;
      }
    }
    __syncthreads();
  }

  // --- one full step of run r ---------------------------------------------
  __device__ static void step(const Tracks &T, const Phys &ph, Smem &sm, uint32_t *words, int r, StepStats &st,
                              bool regrid_only, const mlp::InferSmem *inf) {
    const long long off = T.off[r];
    const double *par = T.par + (size_t)r * gamma_problem::PARAM_WORDS;
    SynchConst sc;
    Hooks::synchrotron_norm(par, &sc.Nalpha, &sc.Nmp, &sc.Nme);
    RunState &R = T.run[r];
    int n = R.ntrack;
    const double t = R.t;
    const int ng = ph.ngst;

    if (Hooks::REGRID) {
      n = regrid_track<Cfg, Hooks, BS>(T.prim, T.N, T.x, T.dx, T.dtl, T.xI, off, n, T.cap[r], ph, par, T.rg,
                                       words, st.splits, st.merges);
      __syncthreads();
    }
    const gamma_problem::HookArgs A{par, ph.gamma_ad, t, R.it, n, ng - 1, n - ng};
    if (regrid_only) {
      if (threadIdx.x == 0) R.ntrack = n;
      __syncthreads();
      return;
    }
    if (Cfg::SHOCK) {  // Cell::resetShock
      for (int i = threadIdx.x; i < n; i += BS) {
        T.sd[off + i] = -1.;
        T.pspec[off + i] = 0.;
        T.shocked[off + i] = 0;
      }
    }
    __syncthreads();

    // stage 1: ghosts, CFL candidates, dt
    edge_geom(T, sm, off, n, ng, 1);
    ghosts(T, ph, A, off, n, sm.edge);
    __syncthreads();
    double m = sweep(T, ph, A, sc, sm, off, n, 1, 0, 0., t, st, inf);
    m = block_min(sm, m);
    const double dt = ph.cfl * m;
    // stage 1 update (the whole Grid::evolve of Timestep/euler.cpp)
    sweep(T, ph, A, sc, sm, off, n, 1, 1, dt, t, st, inf);
    __syncthreads();
    if (!ph.euler) {
      // stage 2
      edge_geom(T, sm, off, n, ng, 2);
      ghosts(T, ph, A, off, n, sm.edge);
      __syncthreads();
      sweep(T, ph, A, sc, sm, off, n, 2, 1, dt, t, st, inf);
      __syncthreads();
      // stage 3
      edge_geom(T, sm, off, n, ng, 3);
      ghosts(T, ph, A, off, n, sm.edge);
      __syncthreads();
      sweep(T, ph, A, sc, sm, off, n, 3, 1, dt, t, st, inf);
      __syncthreads();
    }

    // step-end cell geometry.  RK3: ghosts 0 and n-1 keep the stage-3 ghost
    // copies, cells 1..n-2 span their interfaces (CellGeomFromInterfacePos).
    // Euler: only Cell::update moves cells (iL+1..iR-1); every ghost keeps
    // its stage-1 copy.
    const int iL = ng - 1, iR = n - ng;
    for (int i = threadIdx.x; i < n; i += BS) {
      double gx, gdx;
      if (ph.euler ? (i <= iL || i >= iR) : (i == 0 || i == n - 1)) {
        if (i <= iL) {
          gx = sm.edge[0] - (iL - i + 1) * sm.edge[1];
          gdx = sm.edge[1];
        } else {
          gx = sm.edge[2] + (i - iR + 1) * sm.edge[3];
          gdx = sm.edge[3];
        }
      } else {
        const double xL = T.xI[off + i - 1], xR = T.xI[off + i];
        gx = (xR + xL) / 2.;
        gdx = (xR - xL);
      }
      T.x[off + i] = gx;
      T.dx[off + i] = gdx;
      // radiation_injectParticles on ghost cells (active cells did it in the sweep)
      if (Cfg::SYNCH && (i <= iL || i >= iR)) {
        double prim[NQ];
        load_prim(T, off + i, prim);
        inject_particles<Cfg>(ph, sc, prim, T.shocked[off + i] != 0, T.pspec[off + i]);
        store_prim(T, off + i, prim);
      }
    }
    if (st.status) R.status = st.status;  // any thread; every writer stores the same code
    if (threadIdx.x == 0) {
      R.ntrack = n;
      R.dt = dt;
      R.t = t + dt;
      R.it = R.it + 1;
    }
    st.zone_updates += (unsigned long long)(n - 2 * ng);
    __syncthreads();
  }
};

// Dynamic shared memory: TrackStep::Smem, the regrid bit words (words_bytes),
// then, with GUESS, the tensor-core weights of the learned guess.
// gate (or nullptr): the launch returns at once unless *gate (k_guess_policy)
// chose this kernel, the one with (nonzero) or without (0) the learned guess.
template <class Cfg, class Hooks, int BS, bool GUESS = false, int CPT = 1, int MINB = Cfg::MIN_BLOCKS>
__global__ void __launch_bounds__(BS, MINB)
    track_step_kernel(Tracks T, Phys ph, int nsteps, const int *order, int nruns, int *queue, StepStats *stats,
                      int regrid_only, unsigned words_bytes, const int *gate) {
  if (gate && ((*gate != 0) != GUESS)) return;
  using TS = TrackStep<Cfg, Hooks, BS, GUESS, CPT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  typename TS::Smem &sm = *reinterpret_cast<typename TS::Smem *>(smem_raw);
  uint32_t *words = reinterpret_cast<uint32_t *>(smem_raw + sizeof(typename TS::Smem));
  mlp::InferSmem *inf = nullptr;
  if (GUESS) {
    inf = reinterpret_cast<mlp::InferSmem *>(smem_raw + ((sizeof(typename TS::Smem) + words_bytes + 15u) & ~size_t(15)));
    mlp::load_infer_weights(T.mlp, *inf);
    __syncthreads();
  }
  StepStats st{};
  __shared__ int s_item, s_status;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= nruns) break;
    const int r = order[item];
    for (int k = 0; k < nsteps; ++k) {
      // a run whose step failed stops (block-uniform test)
      if (threadIdx.x == 0) s_status = T.run[r].status;
      __syncthreads();
      const int bad = s_status;
      __syncthreads();
      if (bad != 0) break;
      TS::step(T, ph, sm, words, r, st, regrid_only != 0, inf);
    }
  }
  // fold the per-thread statistics into the launch totals
  __syncthreads();
  if (st.c2p_guesses) atomicAdd(&stats->c2p_guesses, st.c2p_guesses);
  if (st.c2p_poor) atomicAdd(&stats->c2p_poor, st.c2p_poor);
  if (GUESS && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&stats->learned, 1ull);
  if (st.c2p_calls) {
    atomicAdd(&stats->c2p_calls, st.c2p_calls);
    atomicAdd(&stats->c2p_iters, st.c2p_iters);
    atomicAdd(&stats->c2p_fallbacks, st.c2p_fallbacks);
    atomicMax(&stats->c2p_max_iters, st.c2p_max_iters);
  }
  if (threadIdx.x == 0) {
    atomicAdd(&stats->zone_updates, st.zone_updates);
    if (st.splits) atomicAdd(&stats->splits, st.splits);
    if (st.merges) atomicAdd(&stats->merges, st.merges);
  }
  if (st.status) atomicMax(&stats->status, st.status);
}

}  // namespace gb
