// tune.cu — the autotuner: per device and size, the NTT plan (pass widths,
// which fix each pass's radix and its CTA tile of 2^b x G elements) and the
// MSM window width, chosen by timing candidates on the device, installed in
// a process-wide table and saved to / loaded from a text file.
//
// Replaces the fixed choices of the reference (the 1024 x n/1024 split of
// cuda/fft.cu:275-405 and the ln(len) window of cuda/fft.cu:165-172).
// Every plan computes the same DFT and every window the same sum, so a
// choice changes speed only; results stay bit-exact.
//
// File format (one entry per line, '#' comments):
//   device <name with '_' for spaces> <SM count>
//   ntt <log_n> <npass> <b0> <b1> <b2> <b3>
//   msm <log_n> <c>
// Entries follow the last `device` line; zkgpu_tune_load installs them only
// when that line matches the device being loaded for.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "msm.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

namespace zk {
namespace {

std::mutex g_tmu;
std::map<std::pair<int, int>, NttPlan> g_ntt;  // (device, log_n) -> plan
std::map<std::pair<int, int>, int> g_msm;      // (device, log_n) -> c

// primitive 2^log_n-th root of unity: 7^((r - 1) / 2^28) squared 28 - log_n times
host::Fr root_of_unity(int log_n) {
  uint64_t e[4];
  std::memcpy(e, host::R_P, 32);
  e[0] -= 1;  // r - 1 (r is odd)
  for (int k = 0; k < 4; k++) e[k] = (e[k] >> 28) | (k < 3 ? e[k + 1] << 36 : 0);
  host::Fr acc = host::one(), base = host::from_u64(7);
  for (int k = 0; k < 4; k++)
    for (int b = 0; b < 64; b++) {
      if ((e[k] >> b) & 1) acc = host::mul(acc, base);
      base = host::mul(base, base);
    }
  return host::pow_2k(acc, (unsigned)(28 - log_n));
}

std::string device_id(int device, int* sms) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return "";
  std::string n = prop.name;
  for (char& ch : n)
    if (ch == ' ') ch = '_';
  *sms = prop.multiProcessorCount;
  return n;
}

// Candidate plans for log_n: the single pass where it exists, and for
// 2..4 passes every ordering of near-balanced widths (max - min <= 2).
std::vector<NttPlan> ntt_candidates(int log_n) {
  std::vector<NttPlan> out;
  if (log_n <= 2) return out;
  if (log_n <= 11) {
    NttPlan p;
    p.log_n = log_n;
    p.npass = 1;
    p.bits[0] = log_n;
    out.push_back(p);
  }
  const int np_min = std::max(2, (log_n + 10) / 11);
  for (int np = np_min; np <= std::min(NTT_MAX_PASS, np_min + 2); np++) {
    int b[NTT_MAX_PASS] = {3, 3, 3, 3};
    // odometer over widths 3..11
    for (;;) {
      int sum = 0, lo = 99, hi = 0;
      for (int k = 0; k < np; k++) {
        sum += b[k];
        lo = std::min(lo, b[k]);
        hi = std::max(hi, b[k]);
      }
      if (sum == log_n && hi - lo <= 2) {
        NttPlan p;
        p.log_n = log_n;
        p.npass = np;
        for (int k = 0; k < np; k++) p.bits[k] = b[k];
        if (ntt_plan_valid(p)) out.push_back(p);
      }
      int k = 0;
      while (k < np && b[k] == 11) b[k++] = 3;
      if (k == np) break;
      b[k]++;
    }
  }
  return out;
}

__global__ void fill_kernel(fe* a, uint64_t n, uint64_t seed, uint32_t top_mask) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t x = seed + i * 0x9e3779b97f4a7c15ull;
  fe v;
  for (int k = 0; k < 4; k++) {
    x += 0x9e3779b97f4a7c15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    v.w[2 * k] = (uint32_t)z;
    v.w[2 * k + 1] = (uint32_t)(z >> 32);
  }
  v.w[7] &= top_mask;  // 0x0fffffff: below 2^252 < r < q
  a[i] = v;
}

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

// best-of-`reps` time of f() on stream s, after one untimed run
template <class F>
cudaError_t time_best(cudaStream_t s, int reps, F f, float* best) {
  Timer t;
  cudaError_t e = f();
  if (e != cudaSuccess) return e;
  *best = 1e30f;
  for (int r = 0; r < reps; r++) {
    cudaEventRecord(t.a, s);
    e = f();
    if (e != cudaSuccess) return e;
    cudaEventRecord(t.b, s);
    e = cudaEventSynchronize(t.b);
    if (e != cudaSuccess) return e;
    float ms = 0;
    cudaEventElapsedTime(&ms, t.a, t.b);
    *best = std::min(*best, ms);
  }
  return cudaSuccess;
}

void install_ntt(int device, const NttPlan& p) {
  std::lock_guard<std::mutex> lk(g_tmu);
  g_ntt[{device, p.log_n}] = p;
}

// One transform of 2^log_n per trial (tables built per candidate, freed after).
cudaError_t tune_ntt_single(int device, int log_n, int reps, cudaStream_t s, NttPlan* best_plan, float* best_ms) {
  const std::vector<NttPlan> cands = ntt_candidates(log_n);
  if (cands.empty()) return cudaSuccess;
  const size_t n = (size_t)1 << log_n;
  fe *a = nullptr, *tmp = nullptr;
  cudaError_t e = cudaMalloc((void**)&a, n * sizeof(fe));
  if (e == cudaSuccess) e = cudaMalloc((void**)&tmp, n * sizeof(fe));
  if (e == cudaSuccess) {
    fill_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, n, 12345, 0x0fffffffu);
    e = cudaGetLastError();
  }
  const host::Fr w = root_of_unity(log_n);
  *best_ms = 1e30f;
  for (const NttPlan& p : cands) {
    if (e != cudaSuccess) break;
    NttTables t;
    e = ntt_tables_build(&t, p, w, s);
    if (e != cudaSuccess) break;
    float ms = 0;
    e = time_best(s, reps, [&] { return ntt_run(t, a, tmp, nullptr, nullptr, s); }, &ms);
    cudaStreamSynchronize(s);
    ntt_tables_release(&t);
    if (e == cudaSuccess && ms < *best_ms) {
      *best_ms = ms;
      *best_plan = p;
    }
  }
  if (a) cudaFree(a);
  if (tmp) cudaFree(tmp);
  return e;
}

// A batch of 2^log_n transforms filling about 2^22 elements (at most 512
// jobs) through the persistent batch kernel, per candidate plan.
cudaError_t tune_ntt_batched(int device, int log_n, int reps, cudaStream_t s, NttPlan* best_plan, float* best_ms) {
  const std::vector<NttPlan> cands = ntt_candidates(log_n);
  if (cands.empty()) return cudaSuccess;
  const size_t n = (size_t)1 << log_n;
  const size_t jobs = std::max<size_t>(1, std::min<size_t>(512, ((size_t)1 << 22) >> log_n));
  fe* a = nullptr;
  cudaError_t e = cudaMalloc((void**)&a, jobs * n * sizeof(fe));
  if (e == cudaSuccess) {
    fill_kernel<<<(unsigned)((jobs * n + 255) / 256), 256, 0, s>>>(a, jobs * n, 777, 0x0fffffffu);
    e = cudaStreamSynchronize(s);
  }
  const host::Fr w = root_of_unity(log_n);
  std::vector<zkgpu_ntt_job> js(jobs);
  for (size_t j = 0; j < jobs; j++) {
    std::memset(&js[j], 0, sizeof(js[j]));
    js[j].data = reinterpret_cast<uint64_t*>(a + j * n);
    js[j].log_n = (uint32_t)log_n;
    std::memcpy(js[j].omega, w.v, 32);
  }
  NttPlan prev;
  bool had_prev = false;
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    auto it = g_ntt.find({device, log_n});
    if (it != g_ntt.end()) {
      prev = it->second;
      had_prev = true;
    }
  }
  *best_ms = 1e30f;
  for (const NttPlan& p : cands) {
    if (e != cudaSuccess) break;
    install_ntt(device, p);  // the batch builds its passes from the installed plan
    void* b = nullptr;
    int st = zkgpu_ntt_batch_create(device, js.data(), (uint32_t)jobs, &b);
    if (st != ZKGPU_OK) {
      e = cudaErrorUnknown;
      break;
    }
    float ms = 0;
    e = time_best(s, reps, [&] { return zkgpu_ntt_batch_run(b, s) == ZKGPU_OK ? cudaSuccess : cudaErrorUnknown; },
                  &ms);
    cudaStreamSynchronize(s);
    if (e == cudaSuccess && zkgpu_ntt_batch_check(b) != ZKGPU_OK) e = cudaErrorLaunchTimeout;
    zkgpu_ntt_batch_destroy(b);
    if (e == cudaSuccess && ms < *best_ms) {
      *best_ms = ms;
      *best_plan = p;
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    if (had_prev)
      g_ntt[{device, log_n}] = prev;
    else
      g_ntt.erase({device, log_n});
  }
  if (a) cudaFree(a);
  return e;
}

cudaError_t tune_msm(int device, int log_n, int reps, cudaStream_t s, int* best_c, float* best_ms) {
  const uint64_t n = 1ull << log_n;
  fe *sc = nullptr, *bs = nullptr, *out = nullptr;
  cudaError_t e = cudaMalloc((void**)&sc, n * sizeof(fe));
  if (e == cudaSuccess) e = cudaMalloc((void**)&bs, 2 * n * sizeof(fe));
  if (e == cudaSuccess) e = cudaMalloc((void**)&out, 3 * sizeof(fe));
  if (e == cudaSuccess) {
    fill_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(sc, n, 99, 0x0fffffffu);
    fill_kernel<<<(unsigned)((2 * n + 255) / 256), 256, 0, s>>>(bs, 2 * n, 98, 0x0fffffffu);
    e = cudaGetLastError();
  }
  const int d = make_msm_plan(n, 0).c;  // the untuned default for this size
  *best_ms = 1e30f;
  for (int c = std::max(4, d - 2); c <= std::min(16, d + 2) && e == cudaSuccess; c++) {
    float ms = 0;
    e = time_best(s, reps, [&] { return msm_run(sc, bs, n, out, s, c, nullptr); }, &ms);
    if (e == cudaSuccess && ms < *best_ms) {
      *best_ms = ms;
      *best_c = c;
    }
  }
  if (sc) cudaFree(sc);
  if (bs) cudaFree(bs);
  if (out) cudaFree(out);
  return e;
}

}  // namespace

NttPlan tuned_ntt_plan(int device, int log_n) {
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    auto it = g_ntt.find({device, log_n});
    if (it != g_ntt.end()) return it->second;
  }
  return make_ntt_plan(log_n);
}

int tuned_msm_window(int device, int log_n) {
  std::lock_guard<std::mutex> lk(g_tmu);
  auto it = g_msm.find({device, log_n});
  return it == g_msm.end() ? 0 : it->second;
}

}  // namespace zk

using namespace zk;

extern "C" int zkgpu_tune_set_ntt_plan(int device, uint32_t log_n, uint32_t npass, const uint32_t bits[4]) {
  if (device < 0 || log_n > (uint32_t)NTT_MAX_LOG) return ZKGPU_EINVAL;
  if (npass == 0 && log_n > 2) {  // back to the built-in plan
    std::lock_guard<std::mutex> lk(g_tmu);
    g_ntt.erase({device, (int)log_n});
    return ZKGPU_OK;
  }
  if (!bits && npass) return ZKGPU_EINVAL;
  NttPlan p;
  p.log_n = (int)log_n;
  p.npass = (int)npass;
  for (uint32_t k = 0; k < npass && k < (uint32_t)NTT_MAX_PASS; k++) p.bits[k] = (int)bits[k];
  if (npass > (uint32_t)NTT_MAX_PASS || !ntt_plan_valid(p)) return ZKGPU_EINVAL;
  install_ntt(device, p);
  return ZKGPU_OK;
}

extern "C" int zkgpu_tune_get_ntt_plan(int device, uint32_t log_n, uint32_t* npass, uint32_t bits[4]) {
  if (device < 0 || log_n > (uint32_t)NTT_MAX_LOG || !npass || !bits) return ZKGPU_EINVAL;
  const NttPlan p = tuned_ntt_plan(device, (int)log_n);
  *npass = (uint32_t)p.npass;
  for (int k = 0; k < NTT_MAX_PASS; k++) bits[k] = (uint32_t)p.bits[k];
  return ZKGPU_OK;
}

extern "C" int zkgpu_tune_set_msm_window(int device, uint32_t log_n, uint32_t c) {
  if (device < 0 || log_n > 31 || (c != 0 && (c < 4 || c > 16))) return ZKGPU_EINVAL;
  std::lock_guard<std::mutex> lk(g_tmu);
  if (c == 0)
    g_msm.erase({device, (int)log_n});
  else
    g_msm[{device, (int)log_n}] = (int)c;
  return ZKGPU_OK;
}

extern "C" int zkgpu_tune_get_msm_window(int device, uint32_t log_n, uint32_t* c) {
  if (device < 0 || log_n > 31 || !c) return ZKGPU_EINVAL;
  int t = tuned_msm_window(device, (int)log_n);
  *c = (uint32_t)(t ? t : make_msm_plan(1ull << log_n, 0).c);
  return ZKGPU_OK;
}

extern "C" int zkgpu_autotune(int device, uint32_t what, uint32_t log_min, uint32_t log_max, uint32_t reps,
                              double* ms_spent) {
  if (log_min > log_max || log_max > (uint32_t)NTT_MAX_LOG || (what & ~7u) || !what) return ZKGPU_EINVAL;
  if ((what & ZKGPU_TUNE_NTT) && (what & ZKGPU_TUNE_NTT_BATCHED)) return ZKGPU_EINVAL;
  if (reps == 0) reps = 3;
  cudaStream_t s;
  int st = bind_device(device, &s);
  if (st) return st;
  Timer wall;
  cudaEventRecord(wall.a, s);
  cudaError_t e = cudaSuccess;
  for (uint32_t L = log_min; L <= log_max && e == cudaSuccess; L++) {
    if (what & (ZKGPU_TUNE_NTT | ZKGPU_TUNE_NTT_BATCHED)) {
      NttPlan best;
      float ms = 0;
      e = (what & ZKGPU_TUNE_NTT) ? tune_ntt_single(device, (int)L, (int)reps, s, &best, &ms)
                                  : tune_ntt_batched(device, (int)L, (int)reps, s, &best, &ms);
      if (e == cudaSuccess && best.npass > 0) install_ntt(device, best);
    }
    if ((what & ZKGPU_TUNE_MSM) && e == cudaSuccess && L >= 8) {
      int c = 0;
      float ms = 0;
      e = tune_msm(device, (int)L, (int)reps, s, &c, &ms);
      if (e == cudaSuccess && c) {
        std::lock_guard<std::mutex> lk(g_tmu);
        g_msm[{device, (int)L}] = c;
      }
    }
  }
  cudaEventRecord(wall.b, s);
  cudaEventSynchronize(wall.b);
  if (ms_spent) {
    float ms = 0;
    cudaEventElapsedTime(&ms, wall.a, wall.b);
    *ms_spent = ms;
  }
  return status_of("autotune", e);
}

extern "C" int zkgpu_tune_save(int device, const char* path) {
  if (!path) return ZKGPU_EINVAL;
  int sms = 0;
  const std::string id = device_id(device, &sms);
  if (id.empty()) return ZKGPU_ENODEV;
  FILE* f = std::fopen(path, "w");
  if (!f) return ZKGPU_EINVAL;
  std::fprintf(f, "# zkgpu autotuner choices\ndevice %s %d\n", id.c_str(), sms);
  std::lock_guard<std::mutex> lk(g_tmu);
  for (const auto& kv : g_ntt) {
    if (kv.first.first != device) continue;
    const NttPlan& p = kv.second;
    std::fprintf(f, "ntt %d %d %d %d %d %d\n", p.log_n, p.npass, p.bits[0], p.bits[1], p.bits[2], p.bits[3]);
  }
  for (const auto& kv : g_msm)
    if (kv.first.first == device) std::fprintf(f, "msm %d %d\n", kv.first.second, kv.second);
  const bool ok = std::fclose(f) == 0;
  return ok ? ZKGPU_OK : ZKGPU_EINVAL;
}

extern "C" int zkgpu_tune_load(int device, const char* path, uint32_t* loaded) {
  if (!path) return ZKGPU_EINVAL;
  int sms = 0;
  const std::string id = device_id(device, &sms);
  if (id.empty()) return ZKGPU_ENODEV;
  FILE* f = std::fopen(path, "r");
  if (!f) return ZKGPU_EINVAL;
  char line[256];
  bool match = false;
  uint32_t count = 0;
  int status = ZKGPU_OK;
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    char name[200];
    int a, b, c0, c1, c2, c3, nsm;
    if (std::sscanf(line, "device %199s %d", name, &nsm) == 2) {
      match = id == name && nsm == sms;
    } else if (std::sscanf(line, "ntt %d %d %d %d %d %d", &a, &b, &c0, &c1, &c2, &c3) == 6) {
      if (!match) continue;
      const uint32_t bits[4] = {(uint32_t)c0, (uint32_t)c1, (uint32_t)c2, (uint32_t)c3};
      if (a < 0 || b < 0 || zkgpu_tune_set_ntt_plan(device, (uint32_t)a, (uint32_t)b, bits) != ZKGPU_OK) {
        status = ZKGPU_EINVAL;
        break;
      }
      count++;
    } else if (std::sscanf(line, "msm %d %d", &a, &b) == 2) {
      if (!match) continue;
      if (a < 0 || b < 0 || zkgpu_tune_set_msm_window(device, (uint32_t)a, (uint32_t)b) != ZKGPU_OK) {
        status = ZKGPU_EINVAL;
        break;
      }
      count++;
    } else {
      status = ZKGPU_EINVAL;
      break;
    }
  }
  std::fclose(f);
  if (loaded) *loaded = count;
  return status;
}
