// A search from a hint, shared by the 2D step (step2d.cuh) and the test
// suite's host check (selftest.cu).
#pragma once

namespace gb {
namespace d2 {

// The first k in [lo0, hi0) where pred(k) is false, or hi0, for a pred that
// is true up to some k and false after it: searched outwards from the hint h
// (clamped into the range) in steps 1, 2, 4, ..., then by bisection.  Any h
// gives the binary search's k; a hint within d of k takes about 2 log2(d)
// tests instead of log2(hi0 - lo0).
template <class Pred>
__host__ __device__ __forceinline__ int partition_from(int lo0, int hi0, long long h, Pred pred) {
  if (hi0 <= lo0) return lo0;
  const int c = (int)(h < lo0 ? lo0 : (h >= hi0 ? hi0 - 1 : h));
  int lo, hi;  // pred(lo) true or lo = lo0 - 1; pred(hi) false or hi = hi0
  if (pred(c)) {
    lo = c;
    int step = 1;
    hi = c + 1;
    while (hi < hi0 && pred(hi)) {
      lo = hi;
      step <<= 1;
      hi = (hi0 - lo > step) ? lo + step : hi0;
    }
  } else {
    hi = c;
    int step = 1;
    lo = c - 1;
    while (lo >= lo0 && !pred(lo)) {
      hi = lo;
      step <<= 1;
      lo = (hi - lo0 >= step) ? hi - step : lo0 - 1;
    }
  }
  while (hi - lo > 1) {
    const int mid = lo + ((hi - lo) >> 1);
    if (pred(mid)) lo = mid;
    else hi = mid;
  }
  return hi;
}

}  // namespace d2
}  // namespace gb
