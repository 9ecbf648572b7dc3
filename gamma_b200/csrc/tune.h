// Launch-shape variants of the 1D step kernel for the autotuner
// (gamma_gpu_autotune).  Variant 0 is the default (128 threads per run, one
// cell per thread per sweep chunk); variants 1.. change the threads per run
// (the CTA size) and the cells each thread takes per chunk.  Every problem
// module instantiates all of them (problem_module.cuh).  The arithmetic of
// every cell is the same in all of them, so they give identical results; only
// the speed differs.
#pragma once

namespace gb {
namespace tune {

constexpr int kVariants = 8;  // variant 0 included

struct Shape {
  int threads, cells_per_thread;
};

// threads per run and cells per thread of each variant
constexpr Shape kShapes[kVariants] = {{128, 1}, {64, 1}, {256, 1}, {128, 2}, {64, 2}, {128, 4}, {512, 1}, {256, 2}};

// The register cap of each variant keeps the default's resident warps per SM,
// with at least two CTAs of 256 threads: a run's chunk barriers then stall
// half an SM, not all of it (the spherical step, 3 x 128 by default, would
// otherwise get one 256-thread CTA of 232 registers; with two of 128 the BM1D
// sweep runs 8.7% faster, at the same bits).
constexpr int min_blocks(int default_blocks, int threads) {
  const int b = default_blocks * 128 / threads;
  return threads == 256 && b < 2 ? 2 : (b > 0 ? b : 1);
}

}  // namespace tune
}  // namespace gb
