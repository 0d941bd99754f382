// ntt_static.cu — an NTT entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code running while a stream is being
// captured into a CUDA graph, hosts whose device memory is pre-partitioned by
// another runtime that owns every allocation, or real-time paths that forbid
// allocator calls.  zkgpu_ntt_dev_static serves them.  The caller passes the
// data (device memory, transformed in place); the scratch the multi-pass NTT
// needs — the ping-pong buffer and the root / twist tables — lives in the
// file-scope device array below, sized for transforms of up to
// 2^ZKGPU_STATIC_NTT_MAX_LOG elements (about 16.8 MB, held by every GPU that
// loads the library until the process exits).
//
// Sharing rules: every call on a device uses the same array and leaves its
// contents behind.  Nothing in it has to start at zero (the tables are
// rebuilt and the buffer fully overwritten on each call), but two calls whose
// work overlaps on the GPU — different streams without ordering between them,
// or different host threads on one device — race on the array and corrupt
// each other's results.  Serialise them (one stream, or events).
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress, with that device current.  Make that first call
// before any stream capture begins.
#include <cstring>
#include <mutex>

#include "ntt.cuh"
#include "runtime.cuh"

namespace {

constexpr int kMaxLog = ZKGPU_STATIC_NTT_MAX_LOG;
constexpr size_t kBuf = (size_t)1 << kMaxLog;                        // ping-pong buffer
constexpr size_t kTables = ((size_t)1 << kMaxLog) + (1u << 10) + (1u << 12);  // twist + pow + inner tables
constexpr size_t kScratchElems = kBuf + kTables;

static __device__ __align__(256) zk::fe g_static_ntt_scratch[kScratchElems];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
zk::fe* g_addr[kMaxDevices] = {nullptr};

}  // namespace

extern "C" int zkgpu_ntt_dev_static(int device, uint64_t* d_a, uint32_t log_n, const uint64_t omega[4],
                                    void* stream) {
  if (!d_a || !omega) return ZKGPU_EINVAL;
  if (log_n > (uint32_t)kMaxLog) {
    zk::set_last_error("zkgpu_ntt_dev_static: log_n exceeds ZKGPU_STATIC_NTT_MAX_LOG", cudaErrorInvalidValue);
    return ZKGPU_EINVAL;
  }
  zk::host::Fr w;
  std::memcpy(w.v, omega, 32);
  if (!zk::host::is_canonical(w) || !zk::host::is_primitive_root(w, log_n)) return ZKGPU_EINVAL;
  if (device < 0 || device >= kMaxDevices) return ZKGPU_ENODEV;
  ZK_TRY("cudaSetDevice", cudaSetDevice(device));
  zk::fe* base;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_static_ntt_scratch);
      if (e != cudaSuccess) return zk::status_of("cudaGetSymbolAddress(static ntt scratch)", e);
      g_addr[device] = static_cast<zk::fe*>(p);
    }
    base = g_addr[device];
  }
  cudaStream_t s = (cudaStream_t)stream;
  zk::NttTables t;
  ZK_TRY("ntt_tables_fill", zk::ntt_tables_fill(&t, w, (int)log_n, base + kBuf, kTables, s));
  if (t.plan.npass > 0) zk::count_launches((uint64_t)t.plan.npass + 3u * (uint64_t)(t.plan.npass - 1));
  cudaError_t e = zk::ntt_run(t, reinterpret_cast<zk::fe*>(d_a), base, nullptr, nullptr, s);
  zk::count_launches(t.plan.npass > 0 ? t.plan.npass : 1);
  return zk::status_of("zkgpu_ntt_dev_static", e);
}
