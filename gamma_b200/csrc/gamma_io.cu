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
#define GB_HD_OUTLINE __host__ __device__ inline
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
  p.eos_ws = c.eos_wavespeeds;
  p.euler = c.timestep == GAMMA_TS_EULER;
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
  p.eos_ws = c.eos_wavespeeds;
  p.euler = c.timestep == GAMMA_TS_EULER;
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
    if (is_sph(cfg)) prim2cons<RefOrder<CfgSph>>(ph, p, c);
    else prim2cons<RefOrder<CfgCart>>(ph, p, c);
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

// The data lines of a dump (the header skipped).  The reference reads lines
// with fgets into 512 bytes; a longer line is refused here.
bool split_lines(const char *path, std::string &text, std::vector<size_t> &start) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) text.append(chunk, got);
  std::fclose(f);
  size_t pos = text.find('\n');
  if (pos == std::string::npos) return false;  // no header line
  ++pos;
  while (pos < text.size()) {
    size_t e = text.find('\n', pos);
    if (e == std::string::npos) e = text.size();
    if (e - pos + 1 > 511) return false;
    if (e > pos) start.push_back(pos);
    pos = e + 1;
  }
  start.push_back(text.size() + 1);  // sentinel: the end of the last line + 1
  return true;
}

// Parses line k of `text` with parse(buf, row) -> ok on several host threads;
// rows keeps the file's order.
template <class Row, class Parse>
bool parse_rows(const std::string &text, const std::vector<size_t> &start, std::vector<Row> &rows, Parse parse) {
  const long long n = (long long)start.size() - 1;
  rows.resize((size_t)std::max<long long>(n, 0));
  unsigned hw = std::thread::hardware_concurrency();
  const int nt = (int)std::max<long long>(1, std::min<long long>({(long long)(hw ? hw : 1), 32, (n + 16383) / 16384}));
  std::vector<char> ok(nt, 1);
  auto work = [&](int k) {
    char buf[512];
    for (long long r = n * k / nt; r < n * (k + 1) / nt; ++r) {
      const size_t a = start[r], len = std::min(start[r + 1] - 1 - a, sizeof(buf) - 1);
      std::memcpy(buf, text.data() + a, len);
      buf[len] = '\0';
      if (!parse(buf, rows[r])) ok[k] = 0;
    }
  };
  if (nt == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int k = 0; k < nt; ++k) th.emplace_back(work, k);
    for (auto &t : th) t.join();
  }
  return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
}

struct Row1 {
  double t, x, dx, rho, vx, p, trac, gmn, gmx;
  int nact, i;
};

struct Row2 {
  double t, x, y, dx, dy, rho, vx, vy, p, trac, gmn, gmx, gmd, psyn;
  int nact, j, i;
};

}  // namespace

GAMMA_API int gamma_text1d_read(const char *path, const gamma_config_t *cfg, int cap, int *ntrack, long long *it,
                                double *t, double *prim, double *x, double *dx, double *xI) {
  if (!path || !cfg || !ntrack || !prim || !x || !dx || !xI || cfg->nq < 6 || cfg->nq > 10) return GAMMA_ERR_INVALID;
  const int ng = cfg->ngst, nq = cfg->nq;
  if (cap < 2 * ng + 1) return GAMMA_ERR_INVALID;
  std::string text;
  std::vector<size_t> start;
  if (!split_lines(path, text, start)) return GAMMA_ERR_IO;
  const bool synch = cfg->local_synchrotron != 0;
  std::vector<Row1> rows;
  // Data::Data and the values Data::toCell stores (text1d.cpp:17-63)
  const bool parsed = parse_rows(text, start, rows, [&](const char *line, Row1 &r) {
    double dlx, D, sx, tau, Sd, gmin = 0., gmax = 0.;
    const int got =
        synch ? std::sscanf(line, "%le %d %d %le %le %le %le %le %le %le %le %le %le %le %le %le\n", &r.t, &r.nact,
                            &r.i, &r.x, &r.dx, &dlx, &r.rho, &r.vx, &r.p, &D, &sx, &tau, &r.trac, &Sd, &gmin, &gmax)
              : std::sscanf(line, "%le %d %d %le %le %le %le %le %le %le %le %le %le\n", &r.t, &r.nact, &r.i, &r.x,
                            &r.dx, &dlx, &r.rho, &r.vx, &r.p, &D, &sx, &tau, &r.trac);
    if (synch) {
      r.gmn = pow(r.rho, 1. / 3.) / gmin;
      r.gmx = pow(r.rho, 1. / 3.) / gmax;
    }
    return got == (synch ? 16 : 13);
  });
  if (!parsed || rows.empty()) return GAMMA_ERR_IO;
  // Grid::initialise + Cell defaults (FluidState: rho = p = 1, the rest 0)
  for (int q = 0; q < nq; ++q)
    for (int i = 0; i < cap; ++i) prim[(size_t)q * cap + i] = (q == RHO || q == PPP) ? 1. : 0.;
  for (int i = 0; i < cap; ++i) x[i] = dx[i] = 0.;
  int nact = -1;
  for (const Row1 &r : rows) {  // file order; Cinit[i] lands in Ctot[ngst + i]
    if (r.i < 0 || r.i + 2 * ng > cap || r.nact + 2 * ng > cap) return GAMMA_ERR_CAPACITY;
    const int c = ng + r.i;
    x[c] = r.x;
    dx[c] = r.dx;
    prim[(size_t)RHO * cap + c] = r.rho;
    prim[(size_t)UU1 * cap + c] = r.vx;  // VV1: a 3-velocity until prepForRun's v2u
    prim[(size_t)PPP * cap + c] = r.p;
    prim[(size_t)TR1 * cap + c] = r.trac;
    if (synch) {
      prim[(size_t)GMN * cap + c] = r.gmn;
      prim[(size_t)GMX * cap + c] = r.gmx;
    }
    nact = r.nact;
  }
  if (nact < 0) return GAMMA_ERR_IO;
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
  if (t) *t = rows.front().t;
  return GAMMA_OK;
}

GAMMA_API int gamma_text2d_read(const char *path, const gamma_2d_config_t *cfg, int *ntrack, long long *it,
                                double *t, double *theta, double *dtheta, double *prim, double *x, double *dx,
                                double *xI) {
  if (!path || !cfg || !ntrack || !prim || !x || !dx || !xI || cfg->nq != 10) return GAMMA_ERR_INVALID;
  const int ng = cfg->ngst, NJ = cfg->ntheta + 2 * ng, cap = cfg->nmax + 2 * ng;
  const long long NC = (long long)NJ * cap;
  std::string text;
  std::vector<size_t> start;
  if (!split_lines(path, text, start)) return GAMMA_ERR_IO;
  std::vector<Row2> rows;
  // Data::Data and the values Data::toCell stores (text2d.cpp:17-67)
  const bool parsed = parse_rows(text, start, rows, [&](const char *line, Row2 &r) {
    double dlx, dly, D, sx, sy, tau, Sd, gmin, gmax, gmid;
    const int got = std::sscanf(
        line, "%le %d %d %d %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le\n", &r.t,
        &r.nact, &r.j, &r.i, &r.x, &r.y, &r.dx, &r.dy, &dlx, &dly, &r.rho, &r.vx, &r.vy, &r.p, &D, &sx, &sy, &tau,
        &r.trac, &Sd, &gmin, &gmax, &gmid, &r.psyn);
    r.gmn = pow(r.rho, 1. / 3.) / gmin;
    r.gmx = pow(r.rho, 1. / 3.) / gmax;
    r.gmd = pow(r.rho, 1. / 3.) / gmid;
    return got == 24;
  });
  if (!parsed || rows.empty()) return GAMMA_ERR_IO;
  for (int q = 0; q < d2::NQ; ++q)
    for (long long g = 0; g < NC; ++g) prim[q * NC + g] = (q == RHO || q == PPP) ? 1. : 0.;
  for (long long g = 0; g < NC; ++g) x[g] = dx[g] = xI[g] = 0.;
  for (int j = 0; j < NJ; ++j) ntrack[j] = 0;
  for (const Row2 &r : rows) {  // file order; Cinit[j][i] lands in Ctot[j+ngst][i+ngst]
    if (r.j < 0 || r.j >= cfg->ntheta || r.i < 0 || r.i >= cfg->nmax || r.nact > cfg->nmax) return GAMMA_ERR_CAPACITY;
    const int jj = r.j + ng;
    const long long g = (long long)jj * cap + ng + r.i;
    x[g] = r.x;
    dx[g] = r.dx;
    if (theta) theta[r.j] = r.y;
    if (dtheta) dtheta[r.j] = r.dy;
    prim[RHO * NC + g] = r.rho;
    prim[UU1 * NC + g] = r.vx;  // VV1, VV2: 3-velocities until v2u
    prim[UU2 * NC + g] = r.vy;
    prim[PPP * NC + g] = r.p;
    prim[TR1 * NC + g] = r.trac;
    prim[GMN * NC + g] = r.gmn;
    prim[GMX * NC + g] = r.gmx;
    prim[GMD * NC + g] = r.gmd;
    prim[PSN * NC + g] = r.psyn;
    ntrack[jj] = r.nact + 2 * ng;  // reloadFromData (text2d.cpp:127-143)
  }
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
  if (t) *t = rows.front().t;
  return GAMMA_OK;
}
