// Large host <-> device copies of pageable host memory (see host_copy.cu).  Both return when the copy
// is complete; the copy runs on stream s after the work already queued there.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace fluxo {
cudaError_t copy_h2d(void* dDst, const void* hSrc, size_t bytes, cudaStream_t s);
cudaError_t copy_d2h(void* hDst, const void* dSrc, size_t bytes, cudaStream_t s);
}  // namespace fluxo
