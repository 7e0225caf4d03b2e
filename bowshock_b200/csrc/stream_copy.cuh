// Copies between host and device memory ordered on the stream the device work runs on.
//
// The arenas and the network launch every kernel on a stream created with cudaStreamNonBlocking, which does not order
// against the legacy default stream that plain cudaMemcpy uses. A cudaMemcpy from pageable host memory to the device
// may return before its DMA has landed (the host buffer is only staged), and one from the device to the host does not
// wait for kernels on another stream. copy_sync enqueues the copy on the given stream, so it follows the stream's
// earlier work and precedes any later launch on it, and returns once the host buffer may be reused or read: at once
// for pageable memory (cudaMemcpyAsync stages a pageable source before returning, and returns from a copy into pageable
// memory only when it has completed), after a wait for the stream for page-locked memory, whose copies run
// asynchronously.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

static inline cudaError_t copy_sync(cudaStream_t st, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
  const void* host = kind == cudaMemcpyHostToDevice ? src : kind == cudaMemcpyDeviceToHost ? dst : nullptr;
  bool wait = host == nullptr;
  if (host) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, host) == cudaSuccess)
      wait = a.type != cudaMemoryTypeUnregistered;
    else
      (void)cudaGetLastError(), wait = true;
  }
  const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, st);
  if (e != cudaSuccess) return e;
  return wait ? cudaStreamSynchronize(st) : cudaSuccess;
}
