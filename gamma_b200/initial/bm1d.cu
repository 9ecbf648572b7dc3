// Problem module: the 1D spherical Blandford-McKee blast wave of
// src/Initial/Tests/BM1D.cpp, run with spherical1D + rel_sph + radiation_sph.
//
// Per-run parameters: the words of gamma_run_params_t (include/gamma_gpu.h),
// which also carry the normalised synchrotron constants.  The set-up hooks
// (loadParams, initialGeometry, initialValues) run on the host in Python
// (gamma_b200/problems.py, Bm1dSetup), checked bit for bit against the
// reference's own initial state.
#include "problem_module.cuh"

namespace {

using gamma_problem::HookArgs;

GAMMA_HD const gamma_run_params_t &bm_params(const double *par) {
  return *reinterpret_cast<const gamma_run_params_t *>(par);
}

struct BM1D : gamma_problem::Problem {
  static constexpr bool REGRID = true;
  static constexpr int REGRID_WINDOW = 10;  // BM1D.cpp:304: 0 < dist < 10

  // calcBM (BM1D.cpp:62-86): the analytic solution at r (code units) and t
  GAMMA_HD static void calc_bm(const gamma_run_params_t &P, double G, double r_code, double t, double *rho,
                               double *u, double *p) {
    using gb::C_LIGHT;
    using gb::MP;
    using gb::PI_;
    const double r = r_code * P.lNorm;
    const double c5 = C_LIGHT * C_LIGHT * C_LIGHT * C_LIGHT * C_LIGHT;
    double lfacShock2 = P.Etot * (17. - 4. * P.k) / (8. * PI_ * P.n_ext * MP * (t * t * t) * c5);
    double RShock = C_LIGHT * t * (1. - 1. / (1. + 2. * (4. - P.k) * lfacShock2));
    double rhoa = P.n_ext * MP * pow(RShock / P.Rscale, -P.k);
    double pa = rhoa * P.eta * C_LIGHT * C_LIGHT;
    double ha = C_LIGHT * C_LIGHT + pa * G / (G - 1.) / rhoa;
    double pf = 2. / 3. * lfacShock2 * ha * rhoa;
    double lfacf = sqrt(fmax(1., .5 * lfacShock2));
    double Df = 2. * lfacShock2 * rhoa;
    double chi = (1. + 2. * (4. - P.k) * lfacShock2) * (1. - r / (C_LIGHT * t));
    *p = pf * pow(chi, -(17. - 4. * P.k) / (12. - 3. * P.k)) / P.pNorm;
    double lfac = sqrt(lfacf * lfacf / chi + 1);
    double D = Df * pow(chi, -(7. - 2. * P.k) / (4. - P.k));
    *rho = D / lfac / P.rhoNorm;
    *u = C_LIGHT * sqrt(1. - 1. / (lfac * lfac)) * lfac / P.vNorm;
  }

  // userBoundaries (BM1D.cpp:254-274): the BM solution in the inner ghosts
  // while t < t_bm_until
  GAMMA_HD static void user_boundaries(const HookArgs &a, int i, double x, double *prim) {
    const gamma_run_params_t &P = bm_params(a.par);
    if (i <= a.iLbnd && a.t < P.t_bm_until) {
      double rho, u, p;
      calc_bm(P, a.gamma_ad, x, a.t, &rho, &u, &p);
      prim[gamma_problem::RHO] = rho;
      prim[gamma_problem::UU1] = u;
      prim[gamma_problem::PPP] = p;
      prim[gamma_problem::TR1] = 2.;
    }
  }

  // userKinematics (BM1D.cpp:188-246): ghost interfaces move at v_in / v_out
  // (the shock-lag test there ends in vb = vOut, which nothing reads)
  GAMMA_HD static void user_kinematics(const HookArgs &a, int i, double *v) {
    const gamma_run_params_t &P = bm_params(a.par);
    const int ng = a.iLbnd + 1;
    if (i < ng) *v = P.v_in;
    if (i >= a.ntrack - 1 - ng) *v = P.v_out;
  }

  // checkCellForRegrid (BM1D.cpp:277-319): the shock is the rightmost active
  // cell with p > 1.5 eta
  GAMMA_HD static bool regrid_marker(const double *par, const double *prim) {
    return prim[gamma_problem::PPP] > 1.5 * bm_params(par).eta;
  }
  GAMMA_HD static int check_cell_for_regrid(const double *par, double dx, const double *prim, int i, int iS,
                                            double rOut) {
    const gamma_run_params_t &P = bm_params(par);
    double ar = dx / (rOut * P.dth);
    double dist = i - iS;
    if (0 < dist && dist < 10) ar *= 10;
    double lfac = gamma_problem::lorentz_factor(prim[gamma_problem::UU1]);
    if (ar > P.split_AR * P.target_ar / pow(lfac, 3. / 2.)) return gamma_problem::split_;
    if (ar < P.merge_AR * P.target_ar / pow(lfac, 3. / 2.)) return gamma_problem::merge_;
    return gamma_problem::skip_;
  }

  GAMMA_HD static void synchrotron_norm(const double *par, double *Nalpha, double *Nmp, double *Nme) {
    const gamma_run_params_t &P = bm_params(par);
    *Nalpha = P.Nalpha;
    *Nmp = P.Nmp;
    *Nme = P.Nme;
  }
};

static_assert(sizeof(gamma_run_params_t) <= gamma_problem::PARAM_WORDS * sizeof(double), "parameter words");

}  // namespace

GAMMA_PROBLEM_MODULE("bm1d", BM1D, gamma_problem::MODULES_SPHERICAL1D, GAMMA_PROBLEM_BM1D)
