/*
 * gamma_problem.h -- problem modules (the reference's INITIAL files) for the
 * B200 moving-mesh step.
 *
 * In the reference a problem is one src/Initial/... .cpp file that implements
 * the user hooks (README.md:74-89): loadParams, Grid::initialGeometry,
 * Grid::initialValues, Grid::userKinematics, Cell::userSourceTerms,
 * Grid::userBoundaries, Grid::checkCellForRegrid, FluidState::cons2prim_user
 * (declared in src/grid.h:64-98, src/cell.h:58-69, src/fluid.h:18), and the
 * Makefile links exactly one of them (INITIAL = Tests/BM1D, Makefile:1).
 *
 * Here a problem module is one .cu file holding a struct of hooks derived from
 * gamma_problem::Problem.  It is registered under a name with GAMMA_PROBLEM_MODULE
 * (gamma_b200/csrc/problem_module.cuh) and compiled into the library with
 *
 *     make -C gamma_b200/csrc INITIAL="path/to/module.cu ..."
 *
 * next to the built-in modules (gamma_b200/initial/: tube, bm1d, isen1d).  A
 * context selects its module at run time: gamma_config_t.problem =
 * gamma_gpu_problem_id("name").  The step kernel is instantiated for each
 * module, so the per-cell hooks are inlined device code (GAMMA_HD), as the
 * reference's hooks are inlined into its loops.
 *
 * Hook semantics.  Every hook is a static member; gamma_problem::Problem holds the
 * reference's no-op bodies, so a module defines only the hooks it changes.
 *   Set-up (host; gamma_gpu_initial_state runs them, then Grid::prepForRun,
 *   radiation_initGammas and the first updateGhosts, as Simu::initialise):
 *     load_params          loadParams: cells, capacity (nmax), start time
 *     initial_geometry     Grid::initialGeometry for active cell i of ncell
 *     initial_values       Grid::initialValues for one cell: prim with the
 *                          3-velocity in slot UU1 (prepForRun's v2u follows)
 *   Step (device, inside the step kernel):
 *     user_boundaries      Grid::userBoundaries (1d.cpp:244): called for every
 *                          ghost cell after the outflow copy of updateGhosts
 *     user_kinematics      Grid::userKinematics (1d.cpp:749): called for every
 *                          interface after v = VI lambda*; may replace v
 *     user_source_terms    Cell::userSourceTerms (cell.cpp:114): adds to the
 *                          cell's cons * dV after the geometric sources
 *     cons2prim_user       FluidState::cons2prim_user (rel_sph.cpp:304,
 *                          rel_cart.cpp:216): adjusts the recovered rho, p, u
 *                          before the pressure floor
 *     check_cell_for_regrid + regrid_marker
 *                          Grid::checkCellForRegrid (1d.cpp:484-557): the
 *                          decision for the cell now at position i of the live
 *                          track.  The library replays the reference's
 *                          sequential loop exactly; what the hook may read of
 *                          the live track besides the cell itself is given to
 *                          it: iS, the position of the rightmost active cell
 *                          for which regrid_marker is true (iLbnd+1 if none),
 *                          and rOut, the centre of the outermost active cell
 *                          (Ctot[iRbnd-1].G.x).  REGRID = true enables it;
 *                          REGRID_WINDOW bounds how iS may enter.
 *
 * Per-run parameters are gamma_problem::PARAM_WORDS doubles whose meaning the module
 * defines (gamma_gpu_set_params_words).  Hooks are called concurrently for
 * different cells and runs; they must not write anything but their arguments.
 */
#ifndef GAMMA_PROBLEM_H
#define GAMMA_PROBLEM_H

#include <math.h>

#ifdef __CUDACC__
#define GAMMA_HD __host__ __device__ __forceinline__
#else
#define GAMMA_HD inline
#endif

namespace gamma_problem {

enum { skip_ = 0, merge_ = 1, split_ = 2 };            /* environment.h:41 */
enum { RHO = 0, PPP = 1, UU1 = 2, UU2 = 3, TR1 = 4 };  /* primitive slots, environment.h:33-36,75 */
enum { DEN = 0, TAU = 1, SS1 = 2, SS2 = 3 };           /* conserved slots */
enum { GMN = 6, GMX = 7, GMD = 8, PSN = 9 };           /* synchrotron tracers (NUM_Q = 10) */

/* The module set a problem runs with (Makefile GEOMETRY/HYDRO/RADIATION):
 * cartesian + rel_cart without shock detection or synchrotron (NUM_Q = 6), or
 * spherical1D + rel_sph + radiation_sph (NUM_Q = 10), or cartesian + rel_cyl
 * (NUM_Q = 6). */
enum { MODULES_CARTESIAN = 0, MODULES_SPHERICAL1D = 1, MODULES_CARTESIAN_REL_CYL = 2 };

constexpr int PARAM_WORDS = 32;

/* FluidState::lfac (fluid.cpp:10-22) of a 1D state with 4-velocity uu. */
GAMMA_HD double lorentz_factor(double uu) {
  double u = 0.;
  u += uu * uu;
  u = sqrt(u);
  return sqrt(1 + u * u);
}

/* What a step hook may read about its run. */
struct HookArgs {
  const double *par;  /* the run's PARAM_WORDS parameter words */
  double gamma_ad;    /* GAMMA_ (environment.h:53) */
  double t;           /* Simu::t at the start of the step (set-up: the start time) */
  long long it;       /* Simu::it */
  int ntrack;         /* Grid::ntrack: cells including ghosts */
  int iLbnd, iRbnd;   /* Grid::iLbnd, iRbnd: the ghost cells are i <= iLbnd and i >= iRbnd */
};

/* loadParams (s_par of environment.h:92-97). */
struct Setup {
  int ncell;    /* active cells */
  int nmax;     /* capacity in active cells */
  double tini;  /* start time */
};

struct Problem {
  static constexpr bool REGRID = false;
  /* check_cell_for_regrid may depend on i - iS only through whether
   * 0 < i - iS < REGRID_WINDOW (0: not at all); BM1D's window is 10
   * (BM1D.cpp:304) */
  static constexpr int REGRID_WINDOW = 0;

  static Setup load_params(const double *par) {
    (void)par;
    return Setup{0, 0, 0.};
  }
  static void initial_geometry(const HookArgs &a, int i, int ncell, double *x, double *dx) {
    (void)a; (void)i; (void)ncell; (void)x; (void)dx;
  }
  static void initial_values(const HookArgs &a, double x, double dx, double *prim) {
    (void)a; (void)x; (void)dx; (void)prim;
  }
  GAMMA_HD static void user_boundaries(const HookArgs &a, int i, double x, double *prim) {
    (void)a; (void)i; (void)x; (void)prim;
  }
  GAMMA_HD static void user_kinematics(const HookArgs &a, int i, double *v) {
    (void)a; (void)i; (void)v;
  }
  GAMMA_HD static void user_source_terms(const HookArgs &a, double x, double dx, double dV, const double *prim,
                                         double *cons_dV, double dt) {
    (void)a; (void)x; (void)dx; (void)dV; (void)prim; (void)cons_dV; (void)dt;
  }
  GAMMA_HD static void cons2prim_user(const double *par, double *rho, double *p, double *uu) {
    (void)par; (void)rho; (void)p; (void)uu;
  }
  GAMMA_HD static bool regrid_marker(const double *par, const double *prim) {
    (void)par; (void)prim;
    return false;
  }
  GAMMA_HD static int check_cell_for_regrid(const double *par, double dx, const double *prim, int i, int iS,
                                            double rOut) {
    (void)par; (void)dx; (void)prim; (void)i; (void)iS; (void)rOut;
    return skip_;
  }
  /* the normalised synchrotron constants (constants.cpp:12-20 normalizeConstants,
   * called from loadParams), read by the radiation module */
  GAMMA_HD static void synchrotron_norm(const double *par, double *Nalpha, double *Nmp, double *Nme) {
    (void)par;
    *Nalpha = 0.;
    *Nmp = 0.;
    *Nme = 0.;
  }
};

}  /* namespace gamma_problem */

#endif
