// Copies between host and device memory ordered on the stream the device work runs on.
//
// The arenas and the network launch every kernel on a stream created with cudaStreamNonBlocking, which does not order
// against the legacy default stream that plain cudaMemcpy uses. A cudaMemcpy from pageable host memory to the device
// may return before its DMA has landed (the host buffer is only staged), and one from the device to the host does not
// wait for kernels on another stream. copy_sync enqueues the copy on the given stream and waits for that stream, so
// the copy follows the stream's earlier work and has landed before any later launch on it.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

static inline cudaError_t copy_sync(cudaStream_t st, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
  const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}
