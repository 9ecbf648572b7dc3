// Per-track AMR split/merge (Grid::regrid, src/Dimensions/1d.cpp:484-728) with
// the problem module's refinement criterion (Hooks::check_cell_for_regrid, e.g.
// src/Initial/Tests/BM1D.cpp:277-319).
//
// The reference walks the active cells left to right and acts immediately:
// a split inserts a cell (the right half is examined next), a merge removes one
// (a left merge skips the next cell), and the criterion itself reads the live
// track (the outermost active cell and the shock index).  Decisions are
// therefore inherently sequential, but almost every cell is a no-op whose
// decision does not depend on earlier actions.  So:
//   A. all threads evaluate the criterion for every original cell in the
//      original context (bitmasks of split / merge / high-pressure cells);
//   B. one thread replays the loop exactly.  For an untouched original cell the
//      precomputed decision is valid whenever its distance to the shock is the
//      same as in the original context (checked per cell); runs of valid no-op
//      cells are skipped a bitmask word at a time, so the replay costs
//      O(actions + cells/32).  New cells and cells near a moved shock are
//      evaluated in place.  The replay emits the new track as segments
//      (a run of original cells, or one new cell);
//   C. all threads expand the segments into the new track.
#pragma once

#include "physics.cuh"
#include "types.cuh"

namespace gb {

struct RegridScratch {
  double *nprim;                    // [NQS][2N] new cells of run r at 2*off[r] + id
  double *nx, *ndx, *ndtl, *nrifx;  // [2N]
  int *nrif;                        // [2N] right interface: original index, or -1 (then nrifx)
  int *seg_start, *seg_src;         // [4N] at 4*off[r]: output position; src >= 0 original, else -(id+1)
  double *tprim;                    // [NQS][N] compaction target
  double *tx, *tdx, *tdtl, *txI;    // [N]
  long long N;
};

// One cell as seen by the replay: an original (data fetched lazily) or new.
template <class Cfg>
struct RCell {
  double prim[Cfg::NQ];
  double x, dx, dtl;
  double rifx;
  int orig;    // original index, or -1 for a new cell
  int rif;     // right interface: original index, or -1 (position in rifx)
  bool loaded;
};

template <class Cfg>
struct RegridView {
  static constexpr int NQ = Cfg::NQ;
  static constexpr int NQS = Cfg::NQ - 1;
  const double *prim;
  long long N;
  const double *x, *dx, *dtl, *xI;
  long long off;

  __device__ __forceinline__ static int q_of(int s) { return s < 3 ? s : s + 1; }

  __device__ void fetch(RCell<Cfg> &c) const {
    if (c.loaded) return;
    const long long g = off + c.orig;
#pragma unroll
    for (int s = 0; s < NQS; ++s) c.prim[q_of(s)] = prim[s * N + g];
    c.prim[UU2] = 0.;
    c.x = x[g];
    c.dx = dx[g];
    c.dtl = dtl[g];
    c.loaded = true;
  }
  __device__ RCell<Cfg> orig_cell(int k) const {
    RCell<Cfg> c;
    c.orig = k;
    c.rif = k;
    c.rifx = 0.;
    c.loaded = false;
    return c;
  }
};

__device__ __forceinline__ bool bit_of(const uint32_t *w, int k) { return (w[k >> 5] >> (k & 31)) & 1u; }

// first set bit at index >= from and < to, or to
__device__ __forceinline__ int next_set(const uint32_t *w, int from, int to) {
  if (from >= to) return to;
  int wi = from >> 5;
  uint32_t m = w[wi] & (0xffffffffu << (from & 31));
  const int wlast = (to - 1) >> 5;
  while (true) {
    if (m) {
      const int k = (wi << 5) + __ffs(m) - 1;
      return k < to ? k : to;
    }
    if (++wi > wlast) return to;
    m = w[wi];
  }
}

// highest set bit at index in [lo, hi], or -1
__device__ __forceinline__ int last_set(const uint32_t *w, int lo, int hi) {
  if (hi < lo) return -1;
  int wi = hi >> 5;
  uint32_t m = w[wi] & (0xffffffffu >> (31 - (hi & 31)));
  const int wlo = lo >> 5;
  while (true) {
    if (wi == wlo) m &= 0xffffffffu << (lo & 31);
    if (m) return (wi << 5) + 31 - __clz(m);
    if (--wi < wlo) return -1;
    m = w[wi];
  }
}

// Split cell c (between cL and cR) into A | B (Grid::split, 1d.cpp:560-662).
template <class Cfg>
__device__ void split_cells(const RCell<Cfg> &cL, const RCell<Cfg> &c, const RCell<Cfg> &cR, RCell<Cfg> &A,
                            RCell<Cfg> &B) {
  constexpr int NQ = Cfg::NQ;
  const double cenL = make_geom<Cfg>(cL.x, cL.dx).cen;
  const double cen = make_geom<Cfg>(c.x, c.dx).cen;
  const double cenR = make_geom<Cfg>(cR.x, cR.dx).cen;
  double gC[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double gL = (c.prim[q] - cL.prim[q]) / (cen - cenL);
    double gR = (cR.prim[q] - c.prim[q]) / (cenR - cen);
    double gN = (cR.prim[q] - cL.prim[q]) / (cenR - cenL);
    gL = minmod(gL, gN);
    gR = minmod(gR, gN);
    gC[q] = minmod(gL, gR);
  }
  const double x_old = c.x, dl_old = c.dx;
  A.x = x_old - dl_old / 4.;
  B.x = x_old + dl_old / 4.;
  A.dx = dl_old / 2.;
  B.dx = dl_old / 2.;
  const double xL = make_geom<Cfg>(A.x, A.dx).cen;
  const double xR = make_geom<Cfg>(B.x, B.dx).cen;
  const double xI = A.x + A.dx / 2.;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const double Sc = c.prim[q];
    A.prim[q] = Sc + gC[q] * (xL - xI);
    B.prim[q] = Sc + gC[q] * (xR - xI);
  }
  A.prim[UU2] = 0.;
  B.prim[UU2] = 0.;
  // the right half reuses the record of the old right neighbour (1d.cpp:577)
  A.dtl = c.dtl;
  B.dtl = cR.dtl;
  A.rif = -1;
  A.rifx = x_old;
  B.rif = c.rif;
  B.rifx = c.rifx;
  A.orig = B.orig = -1;
  A.loaded = B.loaded = true;
}

// Merge cell c with victim v (Grid::merge, 1d.cpp:665-728).
template <class Cfg, class Hooks>
__device__ void merge_cells(const Phys &ph, const RCell<Cfg> &c, const RCell<Cfg> &v, bool left, RCell<Cfg> &M,
                            C2PStats *cs, const double *par) {
  constexpr int NQ = Cfg::NQ;
  double cc[NQ], cv[NQ], cons[NQ];
  prim2cons<Cfg>(ph, c.prim, cc);
  prim2cons<Cfg>(ph, v.prim, cv);
  const double dV_loc = make_geom<Cfg>(c.x, c.dx).dV;
  const double dV_vic = make_geom<Cfg>(v.x, v.dx).dV;
#pragma unroll
  for (int q = 0; q < NQ; ++q) cons[q] = (cc[q] * dV_loc + cv[q] * dV_vic) / (dV_loc + dV_vic);
  if (left) M.x = ((v.x - v.dx / 2.) + (c.x + c.dx / 2.)) / 2.;
  else M.x = ((v.x + v.dx / 2.) + (c.x - c.dx / 2.)) / 2.;
  M.dx = c.dx + v.dx;
#pragma unroll
  for (int q = 0; q < NQ; ++q) M.prim[q] = c.prim[q];
  cons2prim<Cfg, Hooks>(ph, cons, M.prim, cs, par);
  M.dtl = c.dtl;
  if (left) {
    M.rif = c.rif;
    M.rifx = c.rifx;
  } else {
    M.rif = v.rif;
    M.rifx = v.rifx;
  }
  M.orig = -1;
  M.loaded = true;
}

// Shared-memory words needed by regrid_track for a track of capacity cap.
__host__ __device__ constexpr int regrid_words(int cap) { return (cap + 31) / 32; }

// Regrid one track; returns the new ntrack.  Called by all threads of the CTA.
// words: 4 * regrid_words(cap) uint32 of shared memory.
//
// The criterion: Hooks::check_cell_for_regrid(par, dx, prim, i, iS, rOut) for
// the cell at live position i, where iS is the live position of the rightmost
// active cell marked by Hooks::regrid_marker (iLbnd+1 if none) and rOut the
// centre of the outermost active cell -- the two things BM1D.cpp:285-301 reads
// from the live track.  The criterion may depend on i - iS only through whether
// 0 < i - iS < Hooks::REGRID_WINDOW, so a cell's decision in the original track
// stays valid while that test gives the same answer as in the original track.
template <class Cfg, class Hooks, int BS>
__device__ int regrid_track(double *prim, long long N, double *x, double *dx, double *dtl, double *xI,
                            long long off, int n, int cap, const Phys &ph, const double *par,
                            const RegridScratch &S, uint32_t *words, unsigned long long &nsplit,
                            unsigned long long &nmerge) {
  constexpr int NQ = Cfg::NQ;
  constexpr int NQS = NQ - 1;
  const int ng = ph.ngst, iL = ng - 1, iR0 = n - ng;
  const int nw = regrid_words(cap);
  uint32_t *hpw = words, *spw = words + nw, *mgw = words + 2 * nw, *outhp = words + 3 * nw;
  __shared__ int s_hpmax, s_nnew, s_nseg, s_first;
  const double rOut0 = x[off + iR0 - 1];
  auto load = [&](long long g, double *p) {
#pragma unroll
    for (int s = 0; s < NQS; ++s) p[s < 3 ? s : s + 1] = prim[s * N + g];
    p[UU2] = 0.;
  };

  // ---- A. high-pressure bits and the original shock index
  if (threadIdx.x == 0) s_hpmax = -1;
  for (int w = threadIdx.x; w < 4 * nw; w += BS) words[w] = 0u;
  __syncthreads();
  for (int base = 0; base < n; base += BS) {
    const int k = base + threadIdx.x;
    bool hp = false;
    if (k < n && k >= iL + 1 && k <= iR0 - 1) {
      double p[NQ];
      load(off + k, p);
      hp = Hooks::regrid_marker(par, p);
    }
    const uint32_t b = __ballot_sync(0xffffffffu, hp);
    if ((threadIdx.x & 31) == 0 && k < n) hpw[k >> 5] = b;
    if (hp) atomicMax(&s_hpmax, k);
  }
  __syncthreads();
  const int hpMax = s_hpmax;
  const double iS0 = hpMax >= 0 ? (double)hpMax : (double)(iL + 1);
  // decisions in the original context
  for (int base = 0; base < n; base += BS) {
    const int k = base + threadIdx.x;
    int a = SKIP;
    if (k < n && k >= iL + 1 && k <= iR0 - 1) {
      double p[NQ];
      load(off + k, p);
      a = Hooks::check_cell_for_regrid(par, dx[off + k], p, k, (int)iS0, rOut0);
    }
    const uint32_t bs = __ballot_sync(0xffffffffu, a == SPLIT);
    const uint32_t bm = __ballot_sync(0xffffffffu, a == MERGE);
    if ((threadIdx.x & 31) == 0 && k < n) {
      spw[k >> 5] = bs;
      mgw[k >> 5] = bm;
    }
  }
  __syncthreads();
  // interesting = split | merge (reuse spw|mgw on the fly)

  // ---- B. sequential replay (thread 0)
  if (threadIdx.x == 0) {
    RegridView<Cfg> V{prim, N, x, dx, dtl, xI, off};
    int *seg_start = S.seg_start + 4 * off;
    int *seg_src = S.seg_src + 4 * off;
    const long long noff = 2 * off;
    int nseg = 0, out = 0, nid = 0;
    int seg_next_orig = -2;  // original index that would extend the open segment
    int hp_final = -1;       // rightmost final position (> iL) holding a high-pressure cell
    int first_change = n;    // first output position that differs from the input

    auto emit_orig_range = [&](int k0, int k1) {  // originals [k0, k1) at positions out..
      if (k1 <= k0) return;
      if (!(nseg > 0 && seg_next_orig == k0)) {
        seg_start[nseg] = out;
        seg_src[nseg] = k0;
        ++nseg;
      }
      if (out != k0 && first_change > out) first_change = out;
      const int h = last_set(hpw, k0, k1 - 1);
      if (h >= 0) hp_final = max(hp_final, out + (h - k0));
      out += k1 - k0;
      seg_next_orig = k1;
    };
    auto emit = [&](RCell<Cfg> &c) {
      if (c.orig >= 0) {
        emit_orig_range(c.orig, c.orig + 1);
        return;
      }
      const int id = nid++;
      const long long gid = noff + id;
#pragma unroll
      for (int s = 0; s < NQS; ++s) S.nprim[s * 2 * S.N + gid] = c.prim[s < 3 ? s : s + 1];
      S.nx[gid] = c.x;
      S.ndx[gid] = c.dx;
      S.ndtl[gid] = c.dtl;
      S.nrif[gid] = c.rif;
      S.nrifx[gid] = c.rifx;
      seg_start[nseg] = out;
      seg_src[nseg] = -(id + 1);
      ++nseg;
      seg_next_orig = -2;
      if (first_change > out) first_change = out;
      if (out > iL && Hooks::regrid_marker(par, c.prim)) hp_final = max(hp_final, out);
      ++out;
    };
    auto is_hp = [&](const RCell<Cfg> &c) -> bool {
      if (c.orig >= 0) return bit_of(hpw, c.orig);
      return Hooks::regrid_marker(par, c.prim);
    };

    int ntrack = n, iR = iR0;
    emit_orig_range(0, iL);
    RCell<Cfg> prev = V.orig_cell(iL), curc = V.orig_cell(iL + 1);
    int k = iL + 2;
    int i = iL + 1;
    C2PStats cs;
    while (i <= iR - 1) {
      // current shock index (rightmost high-pressure cell among positions iL+1..iR-1)
      int iS;
      if (hpMax >= k) {
        iS = i + 1 + (hpMax - k);
      } else {
        iS = hp_final;
        if (i - 1 > iL && is_hp(prev)) iS = max(iS, i - 1);
        if (is_hp(curc)) iS = max(iS, i);
        if (iS < 0) iS = iL + 1;
      }
      int action;
      bool valid = false;
      if (curc.orig >= 0) {
        const int dc = i - iS, d0 = curc.orig - (int)iS0;
        const bool mc = 0 < dc && dc < Hooks::REGRID_WINDOW, m0 = 0 < d0 && d0 < Hooks::REGRID_WINDOW;
        if (mc == m0) {
          valid = true;
          action = bit_of(spw, curc.orig) ? SPLIT : (bit_of(mgw, curc.orig) ? MERGE : SKIP);
        }
      }
      if (!valid) {
        V.fetch(curc);
        double rOut;
        if (iR - 1 == i) rOut = curc.x;
        else rOut = x[off + k + (iR - 1 - (i + 1))];
        action = Hooks::check_cell_for_regrid(par, curc.dx, curc.prim, i, iS, rOut);
      } else if (action == SKIP) {
        // skip a run of original no-op cells whose distance to the shock
        // matches the original context (no action moves anything meanwhile)
        const int kc = curc.orig;
        const int delta = i - kc;
        int lim = kc + (iR - i);  // positions i .. iR-1 can be examined
        const bool aligned = (hpMax >= k) || (iS - delta == (int)iS0);
        if (!aligned) {
          // stop before either shock window
          const int w0 = (int)iS0 + 1;
          if (w0 > kc) lim = min(lim, w0);
          else if ((int)iS0 + Hooks::REGRID_WINDOW - 1 > kc) lim = kc + 1;
          const int w1 = iS - delta + 1;
          if (w1 > kc) lim = min(lim, w1);
          else if (iS - delta + Hooks::REGRID_WINDOW - 1 > kc) lim = kc + 1;
        }
        // first original > kc whose precomputed action is not a no-op
        int m = kc + 1;
        while (m < lim) {
          const int ms = next_set(spw, m, lim), mm = next_set(mgw, m, lim);
          m = min(ms, mm);
          break;
        }
        if (m > lim) m = lim;
        const int J = m - kc;  // examined no-op positions i .. i+J-1
        if (J >= 2) {
          emit(prev);
          emit_orig_range(kc, m - 1);
          prev = V.orig_cell(m - 1);
          curc = V.orig_cell(m);
          k = m + 1;
          i += J;
          continue;
        }
      }

      if (action == SPLIT && ntrack < cap - 1) {
        V.fetch(prev);
        V.fetch(curc);
        RCell<Cfg> nxt = V.orig_cell(k);
        V.fetch(nxt);
        RCell<Cfg> A, B;
        split_cells<Cfg>(prev, curc, nxt, A, B);
        emit(prev);
        prev = A;
        curc = B;
        ++ntrack;
        ++iR;
        ++nsplit;
        ++i;
        continue;
      }
      if (action == MERGE && ntrack > 2 * ng + 2) {
        V.fetch(prev);
        V.fetch(curc);
        RCell<Cfg> nxt = V.orig_cell(k);
        V.fetch(nxt);
        const bool left = (prev.dx < nxt.dx && i != ng) || i == iR - 1;
        RCell<Cfg> M;
        if (left) {
          merge_cells<Cfg, Hooks>(ph, curc, prev, true, M, &cs, par);
          emit(M);
          prev = nxt;
          curc = V.orig_cell(k + 1);
        } else {
          merge_cells<Cfg, Hooks>(ph, curc, nxt, false, M, &cs, par);
          emit(prev);
          prev = M;
          curc = V.orig_cell(k + 1);
        }
        k += 2;
        --ntrack;
        --iR;
        ++nmerge;
        ++i;
        continue;
      }
      // no action
      emit(prev);
      prev = curc;
      curc = V.orig_cell(k);
      ++k;
      ++i;
    }
    emit(prev);
    emit(curc);
    emit_orig_range(k, n);
    s_nnew = out;
    s_nseg = nseg;
    s_first = first_change;
  }
  __syncthreads();
  const int nnew = s_nnew, nseg = s_nseg, first = s_first;
  if (first >= nnew && nnew == n) return n;  // nothing moved

  // ---- C. expand the segments into the new track (positions >= first)
  const int *seg_start = S.seg_start + 4 * off;
  const int *seg_src = S.seg_src + 4 * off;
  const long long noff = 2 * off;
  for (int p = first + threadIdx.x; p < nnew; p += BS) {
    int lo = 0, hi = nseg - 1;  // last segment with start <= p
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (seg_start[mid] <= p) lo = mid;
      else hi = mid - 1;
    }
    const int src = seg_src[lo];
    const long long gp = off + p;
    if (src >= 0) {
      const int kk = src + (p - seg_start[lo]);
      const long long gk = off + kk;
#pragma unroll
      for (int s = 0; s < NQS; ++s) S.tprim[s * S.N + gp] = prim[s * N + gk];
      S.tx[gp] = x[gk];
      S.tdx[gp] = dx[gk];
      S.tdtl[gp] = dtl[gk];
      if (p <= nnew - 2) S.txI[gp] = xI[gk];
    } else {
      const long long gid = noff + (-src - 1);
#pragma unroll
      for (int s = 0; s < NQS; ++s) S.tprim[s * S.N + gp] = S.nprim[s * 2 * S.N + gid];
      S.tx[gp] = S.nx[gid];
      S.tdx[gp] = S.ndx[gid];
      S.tdtl[gp] = S.ndtl[gid];
      if (p <= nnew - 2) {
        const int rif = S.nrif[gid];
        S.txI[gp] = rif >= 0 ? xI[off + rif] : S.nrifx[gid];
      }
    }
  }
  __syncthreads();
  for (int p = first + threadIdx.x; p < nnew; p += BS) {
    const long long gp = off + p;
#pragma unroll
    for (int s = 0; s < NQS; ++s) prim[s * N + gp] = S.tprim[s * S.N + gp];
    x[gp] = S.tx[gp];
    dx[gp] = S.tdx[gp];
    dtl[gp] = S.tdtl[gp];
    if (p <= nnew - 2) xI[gp] = S.txI[gp];
  }
  (void)outhp;
  __syncthreads();
  return nnew;
}

}  // namespace gb
