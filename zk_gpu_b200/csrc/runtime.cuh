// runtime.cuh — per-thread device context, error reporting and launch
// accounting shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/zkgpu.h"

namespace zk {

// Thread-local record of the last CUDA failure (zkgpu_last_error()).
void set_last_error(const char* where, cudaError_t e);
void clear_last_error();

// Kernel launches issued from this thread (zkgpu_launch_count()).
void count_launches(uint64_t k);

// Map a cudaError_t to a ZKGPU_* status, recording the message.
int status_of(const char* where, cudaError_t e);

// Make `device` current on this thread and return this thread's work stream
// for it (created once, non-blocking).
int bind_device(int device, cudaStream_t* stream);

// Stream-ordered device allocation from the library's own memory pool on the
// current device (created on first use).  The pool keeps freed memory cached
// for reuse by later calls; the process's default pool, which the caller's
// own allocations may use, is left as the caller configured it.  Free with
// cudaFreeAsync.  zkgpu_release_cached returns the cached memory.
cudaError_t dmalloc(void** ptr, size_t bytes, cudaStream_t s);
// Take `bytes` of device memory into the library pool of the current device
// and keep it there (one block allocated and freed on `s`, then waited for):
// later allocations are carved from retained memory instead of growing the
// pool, which maps new memory on the calling thread (30-135 ms for a 3-6 GB
// request on B200).
cudaError_t reserve_pool(size_t bytes, cudaStream_t s);
// Return the library pool's cached, unused memory on `device` to the system.
cudaError_t trim_pool(int device);
// Copies for the host-buffer entry points, enqueued on `s`.  Pinned host
// memory is copied directly; pageable memory goes through a per-thread ring
// of pinned chunks (staging.cu).  h2d_copy returns once the source is no
// longer needed (pageable) or the copy is enqueued (pinned); d2h_copy on
// pageable memory returns with the data in `dst`, on pinned memory once the
// copy is enqueued.
bool host_pinned(const void* p);
cudaError_t h2d_copy(void* dst, const void* src, size_t n, cudaStream_t s);
cudaError_t d2h_copy(void* dst, const void* src, size_t n, cudaStream_t s);
template <class T>
inline cudaError_t dmalloc(T** ptr, size_t bytes, cudaStream_t s) {
  return dmalloc(reinterpret_cast<void**>(ptr), bytes, s);
}

}  // namespace zk

#define ZK_TRY(where, expr)                                 \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return ::zk::status_of(where, _e); \
  } while (0)
