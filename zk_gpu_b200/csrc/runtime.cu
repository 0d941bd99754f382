// runtime.cu — device binding, streams, pools, error state (see runtime.cuh).
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "runtime.cuh"

namespace zk {

namespace {
thread_local char t_err[256] = {0};
thread_local uint64_t t_launches = 0;
struct ThreadStreams {
  std::vector<cudaStream_t> by_dev;
  ~ThreadStreams() {
    // streams are left to the driver at process exit; destroying them here
    // could run after the CUDA runtime has been torn down.
  }
};
thread_local ThreadStreams t_streams;
std::mutex g_pool_mu;
std::vector<cudaMemPool_t> g_pools;  // the library's pool per device, created on first use
}  // namespace

static cudaError_t library_pool(int device, cudaMemPool_t* out) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if ((int)g_pools.size() <= device) g_pools.resize(device + 1, nullptr);
  if (!g_pools[device]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t thr = UINT64_MAX;  // keep freed blocks for the next call instead of returning them
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    g_pools[device] = pool;
  }
  *out = g_pools[device];
  return cudaSuccess;
}

cudaError_t dmalloc(void** ptr, size_t bytes, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaMemPool_t pool;
  e = library_pool(dev, &pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(ptr, bytes, pool, s);
}

cudaError_t reserve_pool(size_t bytes, cudaStream_t s) {
  void* p = nullptr;
  cudaError_t e = dmalloc(&p, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();  // a failed reservation is not an error of the caller's next call
    return e;
  }
  e = cudaFreeAsync(p, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

cudaError_t trim_pool(int device) {
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (device < (int)g_pools.size()) pool = g_pools[device];
  }
  return pool ? cudaMemPoolTrimTo(pool, 0) : cudaSuccess;
}

void set_last_error(const char* where, cudaError_t e) {
  std::snprintf(t_err, sizeof(t_err), "%s: %s (%d)", where, cudaGetErrorString(e), (int)e);
}
void clear_last_error() { t_err[0] = 0; }
void count_launches(uint64_t k) { t_launches += k; }

int status_of(const char* where, cudaError_t e) {
  if (e == cudaSuccess) return ZKGPU_OK;
  set_last_error(where, e);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the sticky-free allocation error
    return ZKGPU_ENOMEM;
  }
  if (e == cudaErrorInvalidDevice || e == cudaErrorNoDevice) return ZKGPU_ENODEV;
  return ZKGPU_ECUDA;
}

int bind_device(int device, cudaStream_t* stream) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess) return status_of("cudaGetDeviceCount", e);
  if (device < 0 || device >= count) {
    set_last_error("bind_device", cudaErrorInvalidDevice);
    return ZKGPU_ENODEV;
  }
  ZK_TRY("cudaSetDevice", cudaSetDevice(device));
  if ((int)t_streams.by_dev.size() < count) t_streams.by_dev.resize(count, nullptr);
  if (!t_streams.by_dev[device]) {
    cudaStream_t s;
    ZK_TRY("cudaStreamCreate", cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    t_streams.by_dev[device] = s;
  }
  *stream = t_streams.by_dev[device];
  return ZKGPU_OK;
}

}  // namespace zk

extern "C" const char* zkgpu_last_error(void) { return zk::t_err; }

extern "C" uint64_t zkgpu_launch_count(int reset) {
  uint64_t v = zk::t_launches;
  if (reset) zk::t_launches = 0;
  return v;
}

extern "C" const char* zkgpu_version(void) { return "zkgpu-b200 0.1 (sm_100a)"; }
