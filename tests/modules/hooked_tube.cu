// A problem module compiled into the library from outside its sources
// (make -C gamma_b200/csrc INITIAL=../../tests/modules/hooked_tube.cu): a
// planar shock tube whose every user hook acts, the same hooks as the oracle's
// oracle/ref_harness/hooked_tube_cfg.cpp written against the reference's own
// API.  TEST INFRASTRUCTURE: it pins the routing of each hook.
//
// Parameter words: 0 g, 1 p_floor, 2 v_out, 3 split_dx, 4 merge_dx, 5 ncell,
// 6 nmax, 7 xmin, 8 xmax, 9 xmid, 10 rhoL, 11 pL, 12 vL, 13 rhoR, 14 pR, 15 vR,
// 16 reflect, 17 wall (1: on).
#include "problem_module.cuh"

namespace {

using namespace gamma_problem;

struct HookedTube : Problem {
  static constexpr bool REGRID = true;

  static Setup load_params(const double *par) { return Setup{(int)par[5], (int)par[6], 0.}; }
  static void initial_geometry(const HookArgs &a, int i, int ncell, double *x, double *dx) {
    const double X = a.par[8] - a.par[7];
    *x = (double)X * (i + 0.5) / ncell + a.par[7];
    *dx = X / ncell;
  }
  static void initial_values(const HookArgs &a, double x, double dx, double *prim) {
    (void)dx;
    const bool left = x <= a.par[9];
    prim[RHO] = left ? a.par[10] : a.par[13];
    prim[UU1] = left ? a.par[12] : a.par[15];
    prim[PPP] = left ? a.par[11] : a.par[14];
    prim[TR1] = left ? 1. : 2.;
  }
  // a reflecting wall on the left
  GAMMA_HD static void user_boundaries(const HookArgs &a, int i, double x, double *prim) {
    (void)x;
    if (i <= a.iLbnd && a.par[16] != 0.) prim[UU1] = -prim[UU1];
  }
  GAMMA_HD static void user_kinematics(const HookArgs &a, int i, double *v) {
    const int ng = a.iLbnd + 1;
    if (i < ng && a.par[17] != 0.) *v = 0.;
    if (i >= a.ntrack - 1 - ng) *v = a.par[2];
  }
  GAMMA_HD static void user_source_terms(const HookArgs &a, double x, double dx, double dV, const double *prim,
                                         double *cons_dV, double dt) {
    (void)x; (void)dx; (void)dV; (void)prim;
    cons_dV[SS1] -= a.par[0] * cons_dV[DEN] * dt;
  }
  GAMMA_HD static void cons2prim_user(const double *par, double *rho, double *p, double *uu) {
    (void)rho; (void)uu;
    *p = fmax(*p, par[1]);
  }
  GAMMA_HD static int check_cell_for_regrid(const double *par, double dx, const double *prim, int i, int iS,
                                            double rOut) {
    (void)prim; (void)i; (void)iS; (void)rOut;
    if (dx > par[3]) return split_;
    if (dx < par[4]) return merge_;
    return skip_;
  }
};

}  // namespace

GAMMA_PROBLEM_MODULE("hooked_tube", HookedTube, gamma_problem::MODULES_CARTESIAN, -1)
