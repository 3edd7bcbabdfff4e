// Host-to-device copies that have landed when they return. A plain cudaMemcpy from pageable host
// memory may return once its bytes are staged, before the DMA reaches device memory, and it runs
// on the legacy default stream, which the library's non-blocking streams do not wait for: a kernel
// launched afterwards on such a stream could read the destination before the copy lands. These
// wait for the legacy stream, so work launched after them on any stream sees the data.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace lbg {

inline cudaError_t upload_sync(void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  return e == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : e;
}

}  // namespace lbg
