/*
 * The reference's own Tests/BM1D.cpp, unmodified, run through the B200 shim
 * (gamma_b200/shim/simu_b200.cpp, which replaces src/simu.cpp).  TEST
 * INFRASTRUCTURE: the glue a maintainer writes beside an Initial file -- the
 * library's module name and its parameter words, taken from the Initial
 * file's own constants (included here so that its file statics are in scope).
 *
 *   shim_bm1d <out.bin>     runs main.cpp's sequence (mpi_init,
 *                           checkEnvironment, Simu::initialise, Simu::run)
 *                           and writes the final track (GAMMA_SHIM_MAX_STEPS
 *                           bounds the run).
 */
#include "BM1D.cpp"  // src/Initial/Tests/BM1D.cpp (on the include path)

#include <cstdio>

#include "gamma_gpu.h"
#include "mpisetup.h"

extern "C" const char *gamma_shim_problem(double *w, int *n) {
  // gamma_run_params_t: BM1D.cpp's constants, userBoundaries' t < 1e7 and
  // userKinematics' vIn / vOut, and the normalised synchrotron constants
  gamma_run_params_t p = {Etot, n_ext, eta, k, Rscale, rhoNorm, pNorm, lNorm, vNorm, dth, target_ar, split_AR,
                          merge_AR, 1.e7, 0., 1.5, Nalpha_, Nmp_, Nme_};
  const double *pw = reinterpret_cast<const double *>(&p);
  *n = (int)(sizeof(p) / sizeof(double));
  for (int i = 0; i < *n; ++i) w[i] = pw[i];
  return "bm1d";
}

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  mpi_init(&argc, &argv);
  checkEnvironment();
  Simu s;
  s.initialise();
  s.run();
  FILE *f = std::fopen(argv[1], "wb");
  if (!f) return 3;
  const int n = s.grid.ntrack, nq = NUM_Q;
  std::fwrite(&n, sizeof(int), 1, f);
  std::fwrite(&nq, sizeof(int), 1, f);
  std::fwrite(&s.t, sizeof(double), 1, f);
  const long long it = s.it;
  std::fwrite(&it, sizeof(long long), 1, f);
  for (int q = 0; q < nq; ++q)
    for (int i = 0; i < n; ++i) std::fwrite(&s.grid.Ctot[i].S.prim[q], sizeof(double), 1, f);
  for (int i = 0; i < n; ++i) std::fwrite(&s.grid.Ctot[i].G.x[MV], sizeof(double), 1, f);
  for (int i = 0; i < n; ++i) std::fwrite(&s.grid.Ctot[i].G.dx[MV], sizeof(double), 1, f);
  for (int i = 0; i < n - 1; ++i) std::fwrite(&s.grid.Itot[i].x[MV], sizeof(double), 1, f);
  std::fclose(f);
  return 0;
}
