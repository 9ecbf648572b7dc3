// Problem module: the isentropic simple wave of src/Initial/Tests/isen1D.cpp
// (a smooth-flow convergence test: a density bump whose velocity keeps the
// Riemann invariant J- uniform), run with cartesian + rel_cart.
//
// isen1D has no kinematics, boundary, source or regrid hooks
// (isen1D.cpp:116-160).  Its set-up hooks run on the host through
// gamma_gpu_initial_state.  Parameter words (the file-static constants of
// isen1D.cpp:13-24; zero words take those values):
//   0 Nx     cells (3160)           5 v_ref   (0)
//   1 extra  nmax - Nx (50)         6 p_ref   (1e2)
//   2 xmin   (-0.35)                7 alpha   (1)
//   3 xmax   (1)                    8 L       (0.3)
//   4 rho_ref (1)                   9 angle   (0; any value is taken as given)
#include "problem_module.cuh"

namespace {

using gamma_problem::HookArgs;

struct IsenParams {
  int Nx, extra;
  double xmin, xmax, rho_ref, v_ref, p_ref, alpha, L, angle;
};

IsenParams isen_params(const double *par) {
  auto w = [&](int k, double dflt) { return par[k] != 0. ? par[k] : dflt; };
  IsenParams P;
  P.Nx = (int)w(0, 3160.);
  P.extra = (int)w(1, 50.);
  P.xmin = w(2, -0.35);
  P.xmax = w(3, 1.);
  P.rho_ref = w(4, 1.);
  P.v_ref = par[5];
  P.p_ref = w(6, 1.e2);
  P.alpha = w(7, 1.);
  P.L = w(8, 0.3);
  P.angle = par[9];
  return P;
}

// Riemann invariants J+ and J- (isen1D.cpp:52-62)
double Jm(double G, double v, double cs) {
  return (1. / 2. * log((1 + v) / (1 - v)) - 1. / sqrt(G - 1.) * log((sqrt(G - 1) + cs) / (sqrt(G - 1) - cs)));
}

struct Isen1D : gamma_problem::Problem {
  // loadParams (isen1D.cpp:26-34)
  static gamma_problem::Setup load_params(const double *par) {
    const IsenParams P = isen_params(par);
    return gamma_problem::Setup{P.Nx, P.Nx + P.extra, 0.};
  }
  // initialGeometry (isen1D.cpp:36-48)
  static void initial_geometry(const HookArgs &a, int i, int ncell, double *x, double *dx) {
    const IsenParams P = isen_params(a.par);
    const double X = P.xmax - P.xmin;
    *x = (double)X * (i + 0.5) / ncell + P.xmin;
    *dx = X / ncell;
  }
  // initialValues (isen1D.cpp:65-113).  In 1D the reference's y coordinate
  // G.x[y_] reads past G.x[NUM_D] into G.dx[0], the cell width, so y = dx
  // here; the test fabs(y < 0.3) is then true for every cell narrower than 0.3.
  static void initial_values(const HookArgs &a, double x, double dx, double *prim) {
    const IsenParams P = isen_params(a.par);
    const double G = a.gamma_ad;
    double h_ref = 1. + P.p_ref * G / (G - 1.) / P.rho_ref;
    double cs_ref = sqrt(G * P.p_ref / (P.rho_ref * h_ref));
    double Jm_ref = Jm(G, P.v_ref, cs_ref);
    const double y = dx;
    double x_eff = x * cos(P.angle) - y * sin(P.angle);
    double rho, v, p;
    if (fabs(x_eff) < P.L && fabs((double)(y < 0.3))) {
      rho = P.rho_ref * (1. + P.alpha * pow((x_eff / P.L) * (x_eff / P.L) - 1., 4.));
      p = P.p_ref * pow(rho / P.rho_ref, G);
      double h = 1. + p * G / (G - 1.) / rho;
      double cs = sqrt(G * p / (rho * h));
      double temp = exp(2. * Jm_ref) * pow(((sqrt(G - 1.) + cs) / (sqrt(G - 1.) - cs)), (2. / sqrt(G - 1.)));
      v = (temp - 1.) / (temp + 1.);
      prim[gamma_problem::RHO] = rho;
      prim[gamma_problem::PPP] = p;
      prim[gamma_problem::UU1] = v * cos(P.angle);
      prim[gamma_problem::UU2] = v * sin(P.angle);
      prim[gamma_problem::TR1] = 1;
    } else {
      prim[gamma_problem::RHO] = P.rho_ref;
      prim[gamma_problem::PPP] = P.p_ref;
      prim[gamma_problem::UU1] = P.v_ref * cos(P.angle);
      prim[gamma_problem::UU2] = P.v_ref * sin(P.angle);
      prim[gamma_problem::TR1] = 0;
    }
  }
};

}  // namespace

GAMMA_PROBLEM_MODULE("isen1d", Isen1D, gamma_problem::MODULES_CARTESIAN, -1)
