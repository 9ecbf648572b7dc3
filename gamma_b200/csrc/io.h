// Host-side snapshot helpers shared by the 1D and 2D entry points: the
// reference's text columns (src/IO/text1d.cpp, src/IO/text2d.cpp) and the
// exact binary checkpoint of this library.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "gamma_gpu.h"

namespace gb {
namespace io {

// <dir>/phys%010lld.out, the name Grid::printCols gives a dump of iteration it
std::string phys_name(const char *dir, long long it);

// One run of the 1D build as printCols sees it: `prim` row q (slot q) starts at
// prim + q * stride and holds the run's cells 0 .. ntrack-1, ghosts included.
int write_text1d(const char *path, const gamma_config_t &cfg, int ntrack, long long it, double t,
                 const double *prim, long long stride, const double *x, const double *dx);

// The 2D grid: NJ tracks of `cap` cells; theta/dtheta of the active tracks.
int write_text2d(const char *path, const gamma_2d_config_t &cfg, int NJ, int cap, const int *ntrack,
                 const double *theta, const double *dtheta, long long it, double t, const double *prim,
                 const double *x, const double *dx);

// Binary checkpoint: a tagged sequence of raw blocks.  Every block is written
// with its name and byte count and read back only if both match.
class CkptOut {
 public:
  explicit CkptOut(const char *path);
  ~CkptOut();
  bool ok() const { return f_ != nullptr && good_; }
  void block(const char *name, const void *data, size_t bytes);
  int close();  // GAMMA_OK or GAMMA_ERR_IO

 private:
  FILE *f_;
  bool good_ = true;
};

class CkptIn {
 public:
  explicit CkptIn(const char *path);
  ~CkptIn();
  bool ok() const { return f_ != nullptr && good_; }
  // false (and the reader stops) if the next block is not `name` of `bytes`
  bool block(const char *name, void *data, size_t bytes);

 private:
  FILE *f_;
  bool good_ = true;
};

constexpr uint32_t kCkpt1D = 1, kCkpt2D = 2;

// field by field (the structs have padding)
inline bool same_config(const gamma_config_t &a, const gamma_config_t &b) {
  return a.geometry == b.geometry && a.hydro == b.hydro && a.eos == b.eos && a.nq == b.nq &&
         a.shock_detection == b.shock_detection && a.local_synchrotron == b.local_synchrotron &&
         a.problem == b.problem && a.ngst == b.ngst && a.gamma_ad == b.gamma_ad && a.cfl == b.cfl && a.vi == b.vi &&
         a.eos_wavespeeds == b.eos_wavespeeds && a.timestep == b.timestep;
}
inline bool same_config(const gamma_2d_config_t &a, const gamma_2d_config_t &b) {
  return a.ntheta == b.ntheta && a.nmax == b.nmax && a.ngst == b.ngst && a.nq == b.nq && a.eos == b.eos &&
         a.gamma_ad == b.gamma_ad && a.cfl == b.cfl && a.vi == b.vi && a.eos_wavespeeds == b.eos_wavespeeds &&
         a.timestep == b.timestep;
}

}  // namespace io
}  // namespace gb
