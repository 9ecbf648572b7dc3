// Snapshots (include/gamma_gpu.h, gamma_text* and the checkpoint helpers).
//
// Text: the reference's printCols columns, byte for byte, and its resume
// reader (src/IO/text1d.cpp, src/IO/text2d.cpp).  Host code: the formatting is
// the C library's, and D, S, tau come from the same prim2cons the step uses
// (physics.cuh, physics2d.cuh), compiled for the host here.
//
// Binary checkpoint: this library's own exact format (every array that carries
// state from one step to the next, raw), written as tagged blocks.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

// The state conversions are the step's own (physics.cuh, physics2d.cuh),
// compiled here for the host.
#define GB_HD __host__ __device__ inline
#include "io.h"
#include "physics.cuh"
#include "physics2d.cuh"

namespace gb {
namespace io {

std::string phys_name(const char *dir, long long it) {
  char name[64];
  std::snprintf(name, sizeof(name), "phys%010lld.out", it);
  std::string s = dir ? dir : ".";
  if (!s.empty() && s.back() != '/') s += '/';
  return s + name;
}

namespace {

bool is_sph(const gamma_config_t &c) { return c.hydro == GAMMA_HYDRO_REL_SPH; }

Phys phys_1d(const gamma_config_t &c) {
  Phys p;
  p.gamma_ad = c.gamma_ad;
  p.kgam = c.gamma_ad / (c.gamma_ad - 1.);
  p.cfl = c.cfl;
  p.vi = c.vi;
  p.eos = c.eos;
  p.ngst = c.ngst;
  return p;
}

Phys phys_2d(const gamma_2d_config_t &c) {
  Phys p;
  p.gamma_ad = c.gamma_ad;
  p.kgam = c.gamma_ad / (c.gamma_ad - 1.);
  p.cfl = c.cfl;
  p.vi = c.vi;
  p.eos = c.eos;
  p.ngst = c.ngst;
  return p;
}

// radiation_trac2gammae (radiation_sph.cpp:206-214) applied as
// Cell::radiation_apply_trac2gammae does (:234-243): tracer -> gamma_e
double trac2gammae(double trac, double lfac, double rho) {
  const double g = trac * (lfac * rho);
  if (g != 0.) return (lfac * pow(rho, 4. / 3.) / g);
  return 0;
}

// Formats rows 0 .. n-1 with fmt(row, buf, size) -> characters written and
// writes them in order.  Large dumps are formatted by several host threads,
// each into its own buffer; the bytes are those of one thread's loop.
template <class Fmt>
bool write_rows(FILE *f, long long n, Fmt fmt) {
  constexpr int kLine = 640;
  const long long per = 16384;
  unsigned hw = std::thread::hardware_concurrency();
  const int nt = (int)std::max<long long>(1, std::min<long long>({(long long)(hw ? hw : 1), 32, (n + per - 1) / per}));
  std::vector<std::string> out(nt);
  auto work = [&](int k) {
    const long long a = n * k / nt, b = n * (k + 1) / nt;
    std::string &o = out[k];
    o.reserve((size_t)(b - a) * 256);
    char line[kLine];
    for (long long r = a; r < b; ++r) {
      const int len = fmt(r, line, kLine);
      o.append(line, (size_t)std::min(len, kLine - 1));
    }
  };
  if (nt == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int k = 0; k < nt; ++k) th.emplace_back(work, k);
    for (auto &t : th) t.join();
  }
  for (auto &o : out)
    if (!o.empty() && std::fwrite(o.data(), 1, o.size(), f) != o.size()) return false;
  return true;
}

}  // namespace

int write_text1d(const char *path, const gamma_config_t &cfg, int ntrack, long long it, double t,
                 const double *prim, long long stride, const double *x, const double *dx) {
  if (!path || !prim || !x || !dx || cfg.nq < 6 || cfg.nq > 10 || ntrack < 2 * cfg.ngst) return GAMMA_ERR_INVALID;
  FILE *f = std::fopen(path, "w");
  if (!f) return GAMMA_ERR_IO;
  const Phys ph = phys_1d(cfg);
  const int ng = cfg.ngst, nq = cfg.nq;
  const bool synch = cfg.local_synchrotron != 0;
  if (synch) std::fprintf(f, "t nact i x dx dlx rho vx p D sx tau trac Sd gmin gmax\n");
  else std::fprintf(f, "t nact i x dx dlx rho vx p D sx tau trac Sd\n");
  const int nactd = ntrack - 2 * ng;
  const bool ok = write_rows(f, nactd, [&](long long r, char *line, int size) {
    const int i = ng + (int)r;
    double p[10] = {0}, c[10] = {0};
    for (int q = 0; q < nq; ++q) p[q] = prim[q * stride + i];
    // Cell::S.cons at a dump: cons2prim ends with prim2cons (rel_sph.cpp:318)
    if (is_sph(cfg)) prim2cons<CfgSph>(ph, p, c);
    else prim2cons<CfgCart>(ph, p, c);
    const double lfac = lfac_of(p[UU1]);
    // spherical1D and cartesian: dl = dx (spherical1D.cpp:23-33, cartesian.cpp:20-26)
    if (synch) {
      const double gmin = trac2gammae(p[GMN], lfac, p[RHO]);
      const double gmax = trac2gammae(p[GMX], lfac, p[RHO]);
      return std::snprintf(line, size,
                           "%1.15le %d %d %1.15le %1.15le %1.15le %1.15le %1.15le %1.15le %1.15le %1.15le %1.15le "
                           "%1.15le %1.15le %1.15le %1.15le\n",
                           t, nactd, i - ng, x[i], dx[i], dx[i], p[RHO], p[UU1] / lfac, p[PPP], c[DEN], c[SS1],
                           c[TAU], p[TR1], p[TR1 + 1], gmin, gmax);
    }
    return std::snprintf(line, size,
                         "%1.15le %d %d %1.15le %1.15le %1.15le %1.15le %1.15le %1.15le %1.15le %1.15le %1.15le "
                         "%1.15le %1.15le\n",
                         t, nactd, i - ng, x[i], dx[i], dx[i], p[RHO], p[UU1] / lfac, p[PPP], c[DEN], c[SS1], c[TAU],
                         p[TR1], p[TR1 + 1]);
  });
  return (std::fclose(f) == 0 && ok) ? GAMMA_OK : GAMMA_ERR_IO;
}

int write_text2d(const char *path, const gamma_2d_config_t &cfg, int NJ, int cap, const int *ntrack,
                 const double *theta, const double *dtheta, long long it, double t, const double *prim,
                 const double *x, const double *dx) {
  (void)it;
  if (!path || !ntrack || !theta || !dtheta || !prim || !x || !dx || cfg.nq != 10) return GAMMA_ERR_INVALID;
  FILE *f = std::fopen(path, "w");
  if (!f) return GAMMA_ERR_IO;
  const Phys ph = phys_2d(cfg);
  const int ng = cfg.ngst;
  const long long NC = (long long)NJ * cap;
  std::fprintf(f, "t nact j i x y dx dy dlx dly rho vx vy p D sx sy tau trac Sd gmin gmax gmid psyn\n");
  // rows in (j, i) order: start[k] = first row of active track ng + k
  std::vector<long long> start(NJ - 2 * ng + 1, 0);
  for (int j = ng; j < NJ - ng; ++j) start[j - ng + 1] = start[j - ng] + std::max(0, ntrack[j] - 2 * ng);
  const bool ok = write_rows(f, start.back(), [&](long long r, char *line, int size) {
    const int k = (int)(std::upper_bound(start.begin(), start.end(), r) - start.begin()) - 1;
    const int j = ng + k, n = ntrack[j], i = ng + (int)(r - start[k]);
    const double th = theta[j - ng], dth = dtheta[j - ng];
    const long long g = (long long)j * cap + i;
    double p[d2::NQ], c[d2::NQ];
    for (int q = 0; q < d2::NQ; ++q) p[q] = prim[q * NC + g];
    const double rr = x[g];
    d2::prim2cons(ph, p, c, rr);  // cons2prim(G.x[r_]) ends every update (rk3.cpp:183-191)
    const double lf = d2::lfac(p);
    const double gmin = trac2gammae(p[GMN], lf, p[RHO]);
    const double gmax = trac2gammae(p[GMX], lf, p[RHO]);
    const double gmid = trac2gammae(p[GMD], lf, p[RHO]);
    // spherical: dl = (dr, r dtheta) (spherical.cpp:36-47)
    return std::snprintf(line, size,
                         "%1.15le %d %d %d %1.15le %1.15le %1.15le %1.15le %1.15le %le %le %le %le %le %le %le %le "
                         "%le %le %le %le %le %le %le\n",
                         t, n - 2 * ng, j - ng, i - ng, rr, th, dx[g], dth, dx[g], rr * dth, p[RHO], p[UU1] / lf,
                         p[UU2] / lf, p[PPP], c[DEN], c[SS1], c[SS2], c[TAU], p[TR1], p[TR1 + 1], gmin, gmax, gmid,
                         p[PSN]);
  });
  return (std::fclose(f) == 0 && ok) ? GAMMA_OK : GAMMA_ERR_IO;
}

// ---------------------------------------------------------------------------

CkptOut::CkptOut(const char *path) : f_(path ? std::fopen(path, "wb") : nullptr) {
  static const char magic[8] = {'G', 'A', 'M', 'M', 'A', 'B', '2', '\n'};
  if (f_ && std::fwrite(magic, 1, 8, f_) != 8) good_ = false;
}

CkptOut::~CkptOut() {
  if (f_) std::fclose(f_);
}

void CkptOut::block(const char *name, const void *data, size_t bytes) {
  if (!ok()) return;
  char tag[16] = {0};
  std::strncpy(tag, name, sizeof(tag) - 1);
  const uint64_t n = bytes;
  if (std::fwrite(tag, 1, 16, f_) != 16 || std::fwrite(&n, 8, 1, f_) != 1) good_ = false;
  if (good_ && bytes && std::fwrite(data, 1, bytes, f_) != bytes) good_ = false;
}

int CkptOut::close() {
  if (!f_) return GAMMA_ERR_IO;
  const bool fine = good_;
  const int rc = std::fclose(f_);
  f_ = nullptr;
  return (fine && rc == 0) ? GAMMA_OK : GAMMA_ERR_IO;
}

CkptIn::CkptIn(const char *path) : f_(path ? std::fopen(path, "rb") : nullptr) {
  static const char magic[8] = {'G', 'A', 'M', 'M', 'A', 'B', '2', '\n'};
  char m[8];
  if (f_ && (std::fread(m, 1, 8, f_) != 8 || std::memcmp(m, magic, 8) != 0)) good_ = false;
}

CkptIn::~CkptIn() {
  if (f_) std::fclose(f_);
}

bool CkptIn::block(const char *name, void *data, size_t bytes) {
  if (!ok()) return false;
  char tag[16], want[16] = {0};
  std::strncpy(want, name, sizeof(want) - 1);
  uint64_t n = 0;
  if (std::fread(tag, 1, 16, f_) != 16 || std::fread(&n, 8, 1, f_) != 1 || std::memcmp(tag, want, 16) != 0 ||
      n != bytes) {
    good_ = false;
    return false;
  }
  if (bytes && std::fread(data, 1, bytes, f_) != bytes) good_ = false;
  return good_;
}

}  // namespace io
}  // namespace gb

using namespace gb;

#define GAMMA_API extern "C" __attribute__((visibility("default")))

GAMMA_API int gamma_text1d_write(const char *path, const gamma_config_t *cfg, int ntrack, long long it, double t,
                                 const double *prim, long long stride, const double *x, const double *dx) {
  if (!cfg) return GAMMA_ERR_INVALID;
  return io::write_text1d(path, *cfg, ntrack, it, t, prim, stride, x, dx);
}

GAMMA_API int gamma_text2d_write(const char *path, const gamma_2d_config_t *cfg, const int *ntrack,
                                 const double *theta, const double *dtheta, long long it, double t,
                                 const double *prim, const double *x, const double *dx) {
  if (!cfg) return GAMMA_ERR_INVALID;
  const int NJ = cfg->ntheta + 2 * cfg->ngst, cap = cfg->nmax + 2 * cfg->ngst;
  return io::write_text2d(path, *cfg, NJ, cap, ntrack, theta, dtheta, it, t, prim, x, dx);
}

// ---------------------------------------------------------------------------
// Resume readers (Simu::reinitialise without the problem hooks)

namespace {

// openLastSnapshot's iteration: sscanf(name, "phys%ld.h5") on the file name
long long it_of_name(const char *path) {
  const char *base = std::strrchr(path, '/');
  base = base ? base + 1 : path;
  long it = 0;
  if (std::sscanf(base, "phys%ld", &it) != 1) return 0;
  return it;
}

}  // namespace

GAMMA_API int gamma_text1d_read(const char *path, const gamma_config_t *cfg, int cap, int *ntrack, long long *it,
                                double *t, double *prim, double *x, double *dx, double *xI) {
  if (!path || !cfg || !ntrack || !prim || !x || !dx || !xI || cfg->nq < 6 || cfg->nq > 10) return GAMMA_ERR_INVALID;
  const int ng = cfg->ngst, nq = cfg->nq;
  if (cap < 2 * ng + 1) return GAMMA_ERR_INVALID;
  FILE *f = std::fopen(path, "r");
  if (!f) return GAMMA_ERR_IO;
  // Grid::initialise + Cell defaults (FluidState: rho = p = 1, the rest 0)
  for (int q = 0; q < nq; ++q)
    for (int i = 0; i < cap; ++i) prim[(size_t)q * cap + i] = (q == RHO || q == PPP) ? 1. : 0.;
  for (int i = 0; i < cap; ++i) x[i] = dx[i] = 0.;
  const bool synch = cfg->local_synchrotron != 0;
  char line[512];
  int nact = -1, rows = 0, rc = GAMMA_OK;
  double t0 = 0.;
  if (!std::fgets(line, sizeof(line), f)) rc = GAMMA_ERR_IO;  // header
  while (rc == GAMMA_OK && std::fgets(line, sizeof(line), f)) {
    // Data::Data and Data::toCell (text1d.cpp:17-63); Cinit[i] lands in Ctot[ngst + i]
    double tt, xx, ddx, dlx, rho, vx, p, D, sx, tau, trac, Sd = 0., gmin = 0., gmax = 0.;
    int na, i;
    int got = synch ? std::sscanf(line, "%le %d %d %le %le %le %le %le %le %le %le %le %le %le %le %le\n", &tt, &na,
                                  &i, &xx, &ddx, &dlx, &rho, &vx, &p, &D, &sx, &tau, &trac, &Sd, &gmin, &gmax)
                    : std::sscanf(line, "%le %d %d %le %le %le %le %le %le %le %le %le %le\n", &tt, &na, &i, &xx,
                                  &ddx, &dlx, &rho, &vx, &p, &D, &sx, &tau, &trac);
    if (got != (synch ? 16 : 13)) {
      rc = GAMMA_ERR_IO;
      break;
    }
    if (i < 0 || i + 2 * ng > cap - 0 || na + 2 * ng > cap) {
      rc = GAMMA_ERR_CAPACITY;
      break;
    }
    if (rows == 0) t0 = tt;
    const int c = ng + i;
    x[c] = xx;
    dx[c] = ddx;
    prim[(size_t)RHO * cap + c] = rho;
    prim[(size_t)UU1 * cap + c] = vx;  // VV1: a 3-velocity until prepForRun's v2u
    prim[(size_t)PPP * cap + c] = p;
    prim[(size_t)TR1 * cap + c] = trac;
    if (synch) {
      prim[(size_t)GMN * cap + c] = pow(rho, 1. / 3.) / gmin;
      prim[(size_t)GMX * cap + c] = pow(rho, 1. / 3.) / gmax;
    }
    nact = na;
    ++rows;
  }
  std::fclose(f);
  if (rc != GAMMA_OK) return rc;
  if (rows == 0 || nact < 0) return GAMMA_ERR_IO;
  const int n = nact + 2 * ng;
  // Grid::prepForRun: v2u (1d.cpp:934-951) and interfaceGeomFromCellPos (:844-856)
  for (int i = 0; i < n; ++i) {
    double v = 0.;
    const double vv = prim[(size_t)UU1 * cap + i];
    v += vv * vv;
    v = sqrt(v);
    const double lfac = 1. / sqrt(1. - v * v);
    prim[(size_t)UU1 * cap + i] *= lfac;
  }
  const int iL = ng - 1;
  for (int i = 0; i < n - 1; ++i) xI[i] = (i != iL) ? x[i] + dx[i] / 2. : x[i + 1] - dx[i + 1] / 2.;
  *ntrack = n;
  if (it) *it = it_of_name(path);
  if (t) *t = t0;
  return GAMMA_OK;
}

GAMMA_API int gamma_text2d_read(const char *path, const gamma_2d_config_t *cfg, int *ntrack, long long *it,
                                double *t, double *theta, double *dtheta, double *prim, double *x, double *dx,
                                double *xI) {
  if (!path || !cfg || !ntrack || !prim || !x || !dx || !xI || cfg->nq != 10) return GAMMA_ERR_INVALID;
  const int ng = cfg->ngst, NJ = cfg->ntheta + 2 * ng, cap = cfg->nmax + 2 * ng;
  const long long NC = (long long)NJ * cap;
  FILE *f = std::fopen(path, "r");
  if (!f) return GAMMA_ERR_IO;
  for (int q = 0; q < d2::NQ; ++q)
    for (long long g = 0; g < NC; ++g) prim[q * NC + g] = (q == RHO || q == PPP) ? 1. : 0.;
  for (long long g = 0; g < NC; ++g) x[g] = dx[g] = xI[g] = 0.;
  for (int j = 0; j < NJ; ++j) ntrack[j] = 0;
  char line[512];
  int rows = 0, rc = GAMMA_OK;
  double t0 = 0.;
  if (!std::fgets(line, sizeof(line), f)) rc = GAMMA_ERR_IO;
  while (rc == GAMMA_OK && std::fgets(line, sizeof(line), f)) {
    // Data::Data and Data::toCell (text2d.cpp:17-67); Cinit[j][i] lands in Ctot[j+ngst][i+ngst]
    double tt, xx, yy, ddx, ddy, dlx, dly, rho, vx, vy, p, D, sx, sy, tau, trac, Sd, gmin, gmax, gmid, psyn;
    int na, j, i;
    const int got = std::sscanf(
        line, "%le %d %d %d %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le\n", &tt,
        &na, &j, &i, &xx, &yy, &ddx, &ddy, &dlx, &dly, &rho, &vx, &vy, &p, &D, &sx, &sy, &tau, &trac, &Sd, &gmin,
        &gmax, &gmid, &psyn);
    if (got != 24) {
      rc = GAMMA_ERR_IO;
      break;
    }
    if (j < 0 || j >= cfg->ntheta || i < 0 || i >= cfg->nmax || na > cfg->nmax) {
      rc = GAMMA_ERR_CAPACITY;
      break;
    }
    if (rows == 0) t0 = tt;
    const int jj = j + ng;
    const long long g = (long long)jj * cap + ng + i;
    x[g] = xx;
    dx[g] = ddx;
    if (theta) theta[j] = yy;
    if (dtheta) dtheta[j] = ddy;
    prim[RHO * NC + g] = rho;
    prim[UU1 * NC + g] = vx;  // VV1, VV2: 3-velocities until v2u
    prim[UU2 * NC + g] = vy;
    prim[PPP * NC + g] = p;
    prim[TR1 * NC + g] = trac;
    prim[GMN * NC + g] = pow(rho, 1. / 3.) / gmin;
    prim[GMX * NC + g] = pow(rho, 1. / 3.) / gmax;
    prim[GMD * NC + g] = pow(rho, 1. / 3.) / gmid;
    prim[PSN * NC + g] = psyn;
    ntrack[jj] = na + 2 * ng;  // reloadFromData (text2d.cpp:127-143)
    ++rows;
  }
  std::fclose(f);
  if (rc != GAMMA_OK) return rc;
  if (rows == 0) return GAMMA_ERR_IO;
  // the ghost tracks take the edge tracks' lengths (updateGhosts copies the
  // edge tracks into them, text2d.cpp leaves them as initialise made them)
  for (int j = 0; j < ng; ++j) {
    ntrack[j] = ntrack[ng];
    ntrack[NJ - 1 - j] = ntrack[NJ - 1 - ng];
  }
  // Grid::prepForRun on the active tracks: v2u and interfaceGeomFromCellPos;
  // the ghost tracks are the ghost pass's to fill
  for (int j = ng; j < NJ - ng; ++j) {
    const int n = ntrack[j];
    const long long o = (long long)j * cap;
    for (int i = 0; i < n; ++i) {
      double v = 0.;
      const double v1 = prim[UU1 * NC + o + i], v2 = prim[UU2 * NC + o + i];
      v += v1 * v1;
      v += v2 * v2;
      v = sqrt(v);
      const double lfac = 1. / sqrt(1. - v * v);
      prim[UU1 * NC + o + i] *= lfac;
      prim[UU2 * NC + o + i] *= lfac;
    }
    const int iL = ng - 1;
    for (int i = 0; i < n - 1; ++i)
      xI[o + i] = (i != iL) ? x[o + i] + dx[o + i] / 2. : x[o + i + 1] - dx[o + i + 1] / 2.;
  }
  if (it) *it = it_of_name(path);
  if (t) *t = t0;
  return GAMMA_OK;
}
