// Dynamic shared-memory limits of the library's kernels.
//
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) is a per-kernel, per-device
// setting shared by every caller in the process.  Several contexts and entry
// points launch the same kernel with different amounts of shared memory (a
// context sizes the regrid bit words by its largest track), so a plain
// "set to what I need" from one of them would lower the limit below what
// another one launches with.  raise_smem_limit keeps one high-water mark per
// (device, kernel) and only ever raises the attribute.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace gb {

// Make the current device's limit for kernel fn at least bytes.
cudaError_t raise_smem_limit(const void *fn, size_t bytes);

}  // namespace gb
