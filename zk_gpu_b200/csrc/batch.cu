// batch.cu — many NTTs of uneven sizes in ONE persistent launch, replayed
// from a captured CUDA graph.
//
// This is the single-GPU replacement of the reference's job scheduling
// (src/gpulock.rs:133-226 picks a device and the caller then makes one
// synchronous FFI call per job, each with its own malloc / H2D / five
// launches / D2H, cuda/fft.cu:275-405).  Here a batch is built once from job
// descriptors (device-resident data), every pass of every job becomes a run
// of CTA tiles in one level-ordered work list, and a persistent kernel
// (ntt_batch_kernel) drains the list; a graph holding {counter reset, kernel}
// is replayed for each run.
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "ntt.cuh"
#include "runtime.cuh"

namespace zk {

struct NttBatch {
  int device = 0;
  BatchPass* d_passes = nullptr;
  uint32_t npass = 0, total_tiles = 0;
  uint32_t* d_counters = nullptr;  // [0] next, [1] err, [2..] done per pass
  fe* d_tmp = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int grid = 0;
  uint64_t launches_per_run = 2;
  // tables the graph's passes read, held for the batch's lifetime
  std::vector<NttTablesRef> tables;
  std::vector<PowTablesRef> pows;
  ~NttBatch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (d_passes) cudaFree(d_passes);
    if (d_counters) cudaFree(d_counters);
    if (d_tmp) cudaFree(d_tmp);
  }
};

}  // namespace zk

using zk::fe;
namespace hf = zk::host;

static hf::Fr fr_of(const uint64_t v[4]) {
  hf::Fr r;
  std::memcpy(r.v, v, 32);
  return r;
}

extern "C" int zkgpu_ntt_batch_create(int device, const zkgpu_ntt_job* jobs, uint32_t njobs, void** out) {
  if (!out || (njobs && !jobs)) return ZKGPU_EINVAL;
  *out = nullptr;
  cudaStream_t s;
  int st = zk::bind_device(device, &s);
  if (st) return st;
  auto b = std::make_unique<zk::NttBatch>();
  b->device = device;
  // validate and collect per-job tables
  struct JobInfo {
    zk::NttTablesRef t;
    zk::PowTablesRef pre;
    hf::Fr post;
    bool has_post;
    size_t tmp_off;
  };
  std::vector<JobInfo> info(njobs);
  size_t tmp_elems = 0;
  int max_pass = 0;
  for (uint32_t j = 0; j < njobs; j++) {
    const zkgpu_ntt_job& jb = jobs[j];
    if (!jb.data || jb.log_n < 3 || jb.log_n > (uint32_t)zk::NTT_MAX_LOG) return ZKGPU_EINVAL;
    hf::Fr w = fr_of(jb.omega);
    if (!hf::is_canonical(w) || !hf::is_primitive_root(w, jb.log_n)) return ZKGPU_EINVAL;
    cudaError_t e;
    info[j].t = zk::ntt_tables_get(device, w, (int)jb.log_n, s, &e);
    if (!info[j].t) return zk::status_of("ntt_tables_get", e);
    info[j].pre = nullptr;
    if (jb.flags & ZKGPU_JOB_COSET) {
      hf::Fr c = fr_of(jb.coset);
      if (!hf::is_canonical(c)) return ZKGPU_EINVAL;
      info[j].pre = zk::pow_tables_get(device, c, (int)jb.log_n, s, &e);
      if (!info[j].pre) return zk::status_of("pow_tables_get", e);
    }
    info[j].has_post = (jb.flags & ZKGPU_JOB_SCALE) != 0;
    if (info[j].has_post) {
      info[j].post = fr_of(jb.scale);
      if (!hf::is_canonical(info[j].post)) return ZKGPU_EINVAL;
    }
    info[j].tmp_off = tmp_elems;
    if (info[j].t->plan.npass > 1) tmp_elems += (size_t)1 << jb.log_n;
    if (info[j].t->plan.npass > max_pass) max_pass = info[j].t->plan.npass;
    b->tables.push_back(info[j].t);
    if (info[j].pre) b->pows.push_back(info[j].pre);
  }
  if (tmp_elems) ZK_TRY("cudaMalloc(batch scratch)", cudaMalloc((void**)&b->d_tmp, tmp_elems * sizeof(fe)));
  // level-ordered pass list
  std::vector<zk::BatchPass> passes;
  std::vector<uint32_t> prev_index(njobs, ~0u);
  uint64_t tiles = 0;
  for (int lvl = 0; lvl < max_pass; lvl++) {
    for (uint32_t j = 0; j < njobs; j++) {
      const zk::NttTables& t = *info[j].t;
      if (lvl >= t.plan.npass) continue;
      zk::BatchPass bp{};
      const uint64_t ncta = zk::ntt_pass_params(t, lvl, reinterpret_cast<fe*>(jobs[j].data), b->d_tmp + info[j].tmp_off,
                                                info[j].pre.get(), info[j].has_post ? &info[j].post : nullptr, &bp.p);
      bp.B = (uint32_t)t.plan.bits[lvl];
      bp.ntiles = (uint32_t)ncta;
      bp.tile_base = (uint32_t)tiles;
      bp.dep = prev_index[j];
      bp.dep_tiles = bp.dep == ~0u ? 0u : passes[bp.dep].ntiles;
      prev_index[j] = (uint32_t)passes.size();
      passes.push_back(bp);
      tiles += ncta;
    }
  }
  if (tiles >= (1ull << 32)) return ZKGPU_EINVAL;
  b->npass = (uint32_t)passes.size();
  b->total_tiles = (uint32_t)tiles;
  if (b->npass) {
    ZK_TRY("cudaMalloc(batch passes)", cudaMalloc((void**)&b->d_passes, passes.size() * sizeof(zk::BatchPass)));
    ZK_TRY("batch passes H2D", cudaMemcpy(b->d_passes, passes.data(), passes.size() * sizeof(zk::BatchPass),
                                          cudaMemcpyHostToDevice));
  }
  ZK_TRY("cudaMalloc(batch counters)", cudaMalloc((void**)&b->d_counters, (2 + b->npass) * sizeof(uint32_t)));
  ZK_TRY("cudaMemset", cudaMemset(b->d_counters, 0, (2 + b->npass) * sizeof(uint32_t)));
  b->grid = zk::ntt_batch_grid(device);
  // capture {reset counters, persistent kernel} once
  cudaStream_t cap;
  ZK_TRY("cudaStreamCreate", cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaMemsetAsync(b->d_counters, 0, (2 + b->npass) * sizeof(uint32_t), cap);
    if (b->npass)
      zk::ntt_batch_launch(b->d_passes, b->npass, b->total_tiles, b->d_counters, b->d_counters + 2,
                           b->d_counters + 1, b->grid, cap);
    e = cudaStreamEndCapture(cap, &b->graph);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  cudaStreamDestroy(cap);
  if (e != cudaSuccess) return zk::status_of("batch graph", e);
  *out = b.release();
  return ZKGPU_OK;
}

extern "C" int zkgpu_ntt_batch_run(void* handle, void* stream) {
  auto* b = static_cast<zk::NttBatch*>(handle);
  if (!b) return ZKGPU_EINVAL;
  ZK_TRY("cudaSetDevice", cudaSetDevice(b->device));
  ZK_TRY("cudaGraphLaunch", cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  zk::count_launches(b->npass ? 1 : 0);
  return ZKGPU_OK;
}

extern "C" int zkgpu_ntt_batch_check(void* handle) {
  auto* b = static_cast<zk::NttBatch*>(handle);
  if (!b) return ZKGPU_EINVAL;
  ZK_TRY("cudaSetDevice", cudaSetDevice(b->device));
  uint32_t err = 0;
  ZK_TRY("batch err D2H", cudaMemcpy(&err, b->d_counters + 1, 4, cudaMemcpyDeviceToHost));
  return err ? ZKGPU_ETIMEOUT : ZKGPU_OK;
}

extern "C" void zkgpu_ntt_batch_info(void* handle, uint32_t* passes, uint32_t* tiles, int* grid) {
  auto* b = static_cast<zk::NttBatch*>(handle);
  if (!b) return;
  if (passes) *passes = b->npass;
  if (tiles) *tiles = b->total_tiles;
  if (grid) *grid = b->grid;
}

// Failure detection without a fault: a two-pass transform whose second pass
// waits for one tile more than the first pass has, so nothing ever satisfies
// the wait.  The kernel must give up after ~spin_us, record the error and
// return; the call reports ZKGPU_ETIMEOUT and the context stays usable.
extern "C" int zkgpu_selftest_wait_timeout(int device, const uint64_t omega12[4], uint32_t spin_us) {
  if (!omega12 || spin_us == 0 || spin_us > 2000000) return ZKGPU_EINVAL;
  cudaStream_t s;
  int st = zk::bind_device(device, &s);
  if (st) return st;
  const int L = 12;
  hf::Fr w = fr_of(omega12);
  if (!hf::is_canonical(w) || !hf::is_primitive_root(w, L)) return ZKGPU_EINVAL;
  cudaError_t e;
  const zk::NttTablesRef t = zk::ntt_tables_get(device, w, L, s, &e);
  if (!t) return zk::status_of("ntt_tables_get", e);
  if (t->plan.npass != 2) return ZKGPU_EINVAL;
  fe *d = nullptr, *tmp = nullptr;
  zk::BatchPass* dp = nullptr;
  uint32_t* dc = nullptr;
  ZK_TRY("cudaMalloc", cudaMalloc((void**)&d, (2u << L) * sizeof(fe)));
  tmp = d + (1u << L);
  zk::BatchPass bp[2] = {};
  uint64_t tiles = 0;
  for (int k = 0; k < 2; k++) {
    bp[k].ntiles = (uint32_t)zk::ntt_pass_params(*t, k, d, tmp, nullptr, nullptr, &bp[k].p);
    bp[k].B = (uint32_t)t->plan.bits[k];
    bp[k].tile_base = (uint32_t)tiles;
    tiles += bp[k].ntiles;
  }
  bp[0].dep = ~0u;
  bp[1].dep = 0;
  bp[1].dep_tiles = bp[0].ntiles + 1;  // never reached
  int ds;
  cudaDeviceGetAttribute(&ds, cudaDevAttrClockRate, device);  // kHz
  const uint64_t spin = (uint64_t)spin_us * (uint64_t)(ds > 0 ? ds : 2000000) / 1000ull;
  e = cudaMemset(d, 0, (2u << L) * sizeof(fe));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dp, sizeof(bp));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dc, 4 * 4);
  if (e == cudaSuccess) e = cudaMemcpy(dp, bp, sizeof(bp), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dc, 0, 4 * 4);
  if (e == cudaSuccess) e = zk::ntt_batch_launch(dp, 2, (uint32_t)tiles, dc, dc + 2, dc + 1, zk::ntt_batch_grid(device), s, spin);
  uint32_t err = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&err, dc + 1, 4, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (dp) cudaFree(dp);
  if (dc) cudaFree(dc);
  if (e != cudaSuccess) return zk::status_of("selftest_wait_timeout", e);
  return err ? ZKGPU_ETIMEOUT : ZKGPU_OK;
}

extern "C" void zkgpu_ntt_batch_destroy(void* handle) {
  auto* b = static_cast<zk::NttBatch*>(handle);
  if (!b) return;
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  delete b;
}
