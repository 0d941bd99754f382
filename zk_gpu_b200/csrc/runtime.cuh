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
// for it (created once, non-blocking).  The device's default memory pool is
// configured to keep freed memory cached.
int bind_device(int device, cudaStream_t* stream);

}  // namespace zk

#define ZK_TRY(where, expr)                                 \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) return ::zk::status_of(where, _e); \
  } while (0)
