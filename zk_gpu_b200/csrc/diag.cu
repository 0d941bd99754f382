// diag.cu — measurement support compiled into the library:
//  * zkgpu_int_peak: the device's 32-bit integer multiply-add issue rate
//    (independent mad.lo.cc / madc.hi.cc chains on every SM) and the rate of
//    this library's Fr Montgomery product — the denominators of the NTT /
//    MSM roofline, measured live on the same clock as the workload.
//  * per-kernel CUDA-event timing of launches made while profiling is on
//    (zkgpu_prof_*): each timed launch is bracketed by events on the stream
//    it is launched on, with its algorithmic work attached.
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "field.cuh"
#include "prof.cuh"
#include "runtime.cuh"

namespace zk {

// ---------------------------------------------------------------------------
// integer-pipe peak
// ---------------------------------------------------------------------------
// 8 independent 32-bit multiply-add chains per thread (c = c * a + b, each
// step depends on the last, so nothing is hoisted); one IMAD per step.  This
// is the integer pipe's issue peak (64 per SM-clock on sm_100), the
// conservative denominator: carry-chained forms (madc.hi) run slower.
__global__ void imad_peak_kernel(uint32_t* sink, uint32_t iters, uint32_t seed) {
  uint32_t a[8], c[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    a[i] = (seed * (threadIdx.x + 3 * i + 1)) | 1u;
    c[i] = seed ^ (blockIdx.x * 77u + i);
  }
  const uint32_t b = seed | 1u;
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++) c[i] = c[i] * a[i] + b;
  }
  uint32_t acc = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) acc ^= a[i] ^ c[i];
  if (acc == 0x9e3779b9u) sink[blockIdx.x] = acc;  // keep the work observable
}

// Montgomery products with four independent chains per thread.
__global__ void modmul_rate_kernel(uint32_t* sink, uint32_t iters, uint32_t seed) {
  uint32_t x[4][8], y[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    y[i] = (seed * 2654435761u + i) & 0x0fffffffu;
#pragma unroll
    for (int k = 0; k < 4; k++) x[k][i] = (seed ^ (threadIdx.x * 131u + k * 7u + i)) & 0x0fffffffu;
  }
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 4; k++) mul_rp<FrP>(x[k], x[k], y);
  }
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int i = 0; i < 8; i++) acc ^= x[k][i];
  if (acc == 0x9e3779b9u) sink[blockIdx.x] = acc;
}

// ---------------------------------------------------------------------------
// profiling registry
// ---------------------------------------------------------------------------
namespace {
struct Rec {
  cudaEvent_t a, b;
  double work;   // algorithmic modmuls
  double bytes;  // algorithmic bytes
};
std::mutex g_pmu;
bool g_prof_on = false;
std::map<std::string, std::vector<Rec>> g_recs;
std::vector<cudaEvent_t> g_free_events;

cudaEvent_t take_event() {
  if (!g_free_events.empty()) {
    cudaEvent_t e = g_free_events.back();
    g_free_events.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

ProfScope::ProfScope(const char* name, cudaStream_t s, double work, double bytes) : active_(false), s_(s) {
  std::lock_guard<std::mutex> lk(g_pmu);
  if (!g_prof_on) return;
  active_ = true;
  name_ = name;
  work_ = work;
  bytes_ = bytes;
  a_ = take_event();
  b_ = take_event();
  cudaEventRecord(a_, s_);
}

ProfScope::~ProfScope() {
  if (!active_) return;
  cudaEventRecord(b_, s_);
  std::lock_guard<std::mutex> lk(g_pmu);
  g_recs[name_].push_back(Rec{a_, b_, work_, bytes_});
}

}  // namespace zk

extern "C" int zkgpu_int_peak(int device, uint32_t iters, double* imad_per_s, double* modmul_per_s) {
  cudaStream_t s;
  int st = zk::bind_device(device, &s);
  if (st) return st;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint32_t* sink = nullptr;
  ZK_TRY("cudaMalloc", zk::dmalloc((void**)&sink, 4096 * 4, s));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const unsigned blocks = (unsigned)sms * 8, threads = 256;
  // warm-up, then timed
  zk::imad_peak_kernel<<<blocks, threads, 0, s>>>(sink, 64, 12345u);
  cudaEventRecord(e0, s);
  zk::imad_peak_kernel<<<blocks, threads, 0, s>>>(sink, iters, 12345u);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  if (imad_per_s) *imad_per_s = (double)blocks * threads * iters * 8.0 / (ms * 1e-3);
  const uint32_t mm_iters = iters / 16 > 0 ? iters / 16 : 1;
  zk::modmul_rate_kernel<<<blocks, threads, 0, s>>>(sink, 4, 777u);
  cudaEventRecord(e0, s);
  zk::modmul_rate_kernel<<<blocks, threads, 0, s>>>(sink, mm_iters, 777u);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  if (modmul_per_s) *modmul_per_s = (double)blocks * threads * mm_iters * 4.0 / (ms * 1e-3);
  zk::count_launches(4);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(sink, s);
  return zk::status_of("int_peak", cudaStreamSynchronize(s));
}

extern "C" void zkgpu_prof_enable(int on) {
  std::lock_guard<std::mutex> lk(zk::g_pmu);
  zk::g_prof_on = on != 0;
}

extern "C" void zkgpu_prof_reset(void) {
  std::lock_guard<std::mutex> lk(zk::g_pmu);
  for (auto& kv : zk::g_recs)
    for (auto& r : kv.second) {
      zk::g_free_events.push_back(r.a);
      zk::g_free_events.push_back(r.b);
    }
  zk::g_recs.clear();
}

// Writes up to `cap` lines "name launches total_ms work bytes\n" into buf.
// Synchronises on the recorded events.  Returns the number of kernels.
extern "C" int zkgpu_prof_read(char* buf, uint64_t cap) {
  std::lock_guard<std::mutex> lk(zk::g_pmu);
  std::string out;
  int n = 0;
  for (auto& kv : zk::g_recs) {
    double ms_total = 0, work = 0, bytes = 0;
    for (auto& r : kv.second) {
      cudaEventSynchronize(r.b);
      float ms = 0;
      cudaEventElapsedTime(&ms, r.a, r.b);
      ms_total += ms;
      work += r.work;
      bytes += r.bytes;
    }
    char line[256];
    std::snprintf(line, sizeof(line), "%s %zu %.6f %.6e %.6e\n", kv.first.c_str(), kv.second.size(), ms_total, work,
                  bytes);
    out += line;
    n++;
  }
  if (buf && cap) {
    std::strncpy(buf, out.c_str(), cap - 1);
    buf[cap - 1] = 0;
  }
  return n;
}
