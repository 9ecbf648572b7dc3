/*
 * CPU restatement of GAMMA's 1D moving-mesh relativistic hydro step.
 *
 * TEST INFRASTRUCTURE -- the oracle.  Only tests/, the smoke check and
 * bench.py's CPU-baseline leg load liboracle.so, and only as the checker (or
 * the timed CPU port).  The product never calls it.
 *
 * It restates, in plain C and with the same floating-point operation order,
 * the reference's 1D path: src/Hydro/rel_sph.cpp, src/Hydro/rel_cart.cpp,
 * src/Solver/hllc.cpp, src/cell.cpp, src/interface.cpp,
 * src/Geometry/{spherical1D,cartesian}.cpp, src/Dimensions/1d.cpp,
 * src/Timestep/rk3.cpp, src/Radiation/radiation_sph.cpp, src/simu.cpp, with the
 * problem hooks of src/Initial/Tests/BM1D.cpp (parameterised) and of a planar
 * shock tube (src/Initial/Tests/1DST.cpp).  Compiled with the same flags as the
 * reference build in oracle/_ref it reproduces it bit for bit; tests/ checks
 * that.  The pressure root finder is Brent's zeroin (brent.c) standing in for
 * GSL, which the reference links but does not vendor.
 */
#ifndef GAMMA_ORACLE_H
#define GAMMA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define OC_NQ_MAX 10

enum { OC_GEOM_SPHERICAL1D = 0, OC_GEOM_CARTESIAN = 1 };
enum { OC_HYDRO_REL_SPH = 0, OC_HYDRO_REL_CART = 1 };
enum { OC_EOS_IDEAL = 0, OC_EOS_SYNGE = 1 };
enum { OC_PROBLEM_BM1D = 0, OC_PROBLEM_TUBE = 1 };

/* Run configuration: the reference's compile-time switches
 * (src/environment.h:46-66) and the problem parameters as run-time values. */
typedef struct {
  int geometry;
  int hydro;
  int eos;
  int nq;                 /* NUM_Q: 10 with local synchrotron, 6 without */
  int shock_detection;
  int local_synchrotron;
  int problem;
  int ngst, ncell, nmax;
  double gamma_ad, cfl, vi;
  /* BM1D (src/Initial/Tests/BM1D.cpp:10-56) */
  double n0, eta, Etot, n_ext, tinit, lfac_shock2, lorentz_mode, Rscale, k;
  double grid_log, r_lo, r_hi, dth, target_ar, split_AR, merge_AR, t_bm_until, v_in, v_out;
  /* planar tube */
  double xmin, xmax, xmid, rhoL, pL, vL, trL, rhoR, pR, vR, trR;
  /* relative bracket width at which the pressure root search stops: 1e-13 in
   * the reference (rel_sph.cpp:281); smaller values give a tighter oracle */
  double c2p_epsrel;
  /* 1: Gamma_eff of each state in the wave speeds and the shock detector too
   * (the reference uses GAMMA_ there whatever the EOS; 0 restates it) */
  int eos_wavespeeds;
  /* Grid::evolve: 0 the SSP-RK3 of src/Timestep/rk3.cpp:13-95, 1 the single
   * Grid::update of src/Timestep/euler.cpp:12-19 */
  int timestep;
} oc_config;

typedef struct oc_sim oc_sim;

void oc_config_bm1d_defaults(oc_config *c);
void oc_config_tube_defaults(oc_config *c);

oc_sim *oc_create(const oc_config *cfg);
void oc_destroy(oc_sim *s);
/* Simu::initialise + the pre-loop updateGhosts of Simu::run. */
int oc_init(oc_sim *s);
/* n iterations of the Simu::run loop body.  Returns 0, or the reference's exit
 * code (30: negative CFL candidate) if a step would have ended the process. */
int oc_step(oc_sim *s, int n);
int oc_regrid(oc_sim *s);
/* t, dt, it, ntrack, nact, iLbnd, iRbnd, capacity, tstart, RShock(ls), Nalpha, Nmp, Nme,
 * rhoNorm, pNorm, lNorm, lfacShock2 */
void oc_scalars(const oc_sim *s, double *out);
int oc_snapshot(const oc_sim *s, double *prim, double *x, double *dx, double *dt_loc, double *sd,
                double *pspec, double *shocked, double *xI, int cap);
int oc_load(oc_sim *s, int ntrack, const double *prim, const double *x, const double *dx,
            const double *dt_loc, const double *xI, int cap, double t, long it);

/* Per-state kernels, layout [q*n + k]. */
void oc_cons2prim(const oc_sim *s, double *cons, double *prim, const double *r, int n, int *iters);
void oc_prim2cons(const oc_sim *s, const double *prim, double *cons, const double *r, int n);
void oc_riemann(const oc_sim *s, const double *primL, const double *primR, const double *x,
                const double *v, int v_given, double *lam, double *flux, int n);
/* Analytic Blandford-McKee primitives (rho, u, p) at radius r (ls) and time t (s). */
void oc_bm_profile(const oc_sim *s, const double *r, int n, double t, double *rho, double *u,
                   double *p);

#ifdef __cplusplus
}
#endif

#endif
