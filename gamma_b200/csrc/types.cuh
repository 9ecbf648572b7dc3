// Per-run parameter and state records shared by the kernels and the C-ABI.
#pragma once

#include <cstdint>

namespace gb {

// Problem parameters of one run: the Blandford-McKee hooks of
// src/Initial/Tests/BM1D.cpp (calcBM, userKinematics, checkCellForRegrid) and
// the normalised synchrotron constants of src/constants.cpp:12-20.  Unused by
// problems without hooks (planar tubes).
struct RunParams {
  double Etot, n_ext, eta, k, Rscale;
  double rhoNorm, pNorm, lNorm, vNorm;
  double dth, target_ar, split_AR, merge_AR;
  double t_bm_until, v_in, v_out;
  double Nalpha, Nmp, Nme;
};

// Scalars of one run (Simu::t, dt, it and Grid::ntrack).
struct RunState {
  int ntrack;
  int status;  // 0, or the reference's exit code (30: negative CFL candidate)
  double t, dt;
  long long it;
};

}  // namespace gb
