#pragma once
#include <cstddef>

#include <cuda_runtime.h>

namespace cgfdm {
// Copies `bytes` from pageable host memory to the device, pipelined through
// pinned staging slots by several host threads when large; returns when the
// data is on the device (after the work already queued on `st`).
cudaError_t upload_h2d(void *dst, const void *src, size_t bytes, int device, cudaStream_t st);
}  // namespace cgfdm
