// server.cu — the serving loop: continuous batching of NTT / LDE / MSM jobs
// on one GPU with HBM-budget admission (declared in include/zkgpu.h).
//
// Threads: callers submit (non-blocking) and wait; a scheduler thread admits
// jobs in arrival order while they fit the budget and launches everything it
// admitted as one "wave": all NTT and LDE passes of the wave go into a single
// persistent batch launch (ntt_batch_kernel), MSMs run on a second stream
// against resident base sets; copies are enqueued on the same streams.  A
// completion thread retires waves in order, releases their memory to the
// budget (which wakes the scheduler: new arrivals are admitted while earlier
// waves still run, so their work overlaps on the device) and wakes waiters.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "admission.hpp"
#include "host_field.hpp"
#include "msm.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

namespace zk {

namespace {
using clk = std::chrono::steady_clock;

// Device memory one MSM job of n points holds in flight when it runs alone:
// its scalars, its window sums and the pass's scratch (resident bases are
// already in the curve arithmetic's form, so nothing is converted).
uint64_t msm_job_bytes(uint64_t n, int device) {
  return n * 32 + MSM_MAX_WINDOWS * 128ull + msm_scratch_bytes(n, 1, n, true, false, device);
}

host::Fr fr_of(const uint64_t v[4]) {
  host::Fr r;
  std::memcpy(r.v, v, 32);
  return r;
}

struct JobRec {
  uint64_t ticket = 0;
  zkgpu_job job{};
  uint64_t bytes = 0;
  clk::time_point t_submit, t_done;
  int status = -1;  // -1 in progress
  uint64_t* msm_out = nullptr;  // slot in the wave's pinned mailbox
  cudaEvent_t done_ev = nullptr;  // after this job's result copy (its completion on the GPU side)
  bool retired = false;           // its wave retired (memory released)
  bool taken = false;             // a waiter collected the result
  bool early_failed = false;      // its result is not good: reported at retirement
};

struct Wave {
  std::vector<JobRec*> jobs;
  cudaStream_t s_ntt = nullptr, s_msm = nullptr;
  cudaEvent_t ev_ntt = nullptr, ev_msm = nullptr;
  std::vector<BatchPass> passes;  // host copy kept alive for the async upload
  std::vector<std::shared_ptr<const void>> tables;  // tables the wave's passes read, held until it retires
  uint64_t* mailbox = nullptr;    // pinned: [0] batch error flag, then kMsmSlotWords per MSM job
  BatchPass* pass_stage = nullptr;  // pinned upload buffer of this wave's stream slot (kPassStage entries)
  uint64_t extra_bytes = 0;       // budget taken beyond the jobs' footprints (merged MSM passes)
  int status = ZKGPU_OK;
};

struct BaseSet {
  fe* d = nullptr;
  uint64_t n = 0;
};

}  // namespace

class Server {
 public:
  Server(int dev, uint64_t budget, uint32_t max_wave) : device_(dev), adm_(budget), max_wave_(max_wave ? max_wave : 256) {
    // waves started with whatever is pending (see sched_loop); ZKGPU_SERVER_EAGER_WAVES overrides
    const char* v = std::getenv("ZKGPU_SERVER_EAGER_WAVES");
    if (v && *v) eager_waves_ = std::max(1, std::min(kStreams, std::atoi(v)));
  }

  int start() {
    ZK_TRY("cudaSetDevice", cudaSetDevice(device_));
    for (int i = 0; i < kStreams; i++) {
      ZK_TRY("cudaStreamCreate", cudaStreamCreateWithFlags(&s_ntt_[i], cudaStreamNonBlocking));
      ZK_TRY("cudaStreamCreate", cudaStreamCreateWithFlags(&s_msm_[i], cudaStreamNonBlocking));
    }
    grid_ = ntt_batch_grid(device_);
    // take the budget's memory into the library pool now, capped by what the
    // device has free less a margin for the process's other allocations:
    // waves then carve their buffers from retained memory instead of growing
    // the pool while the GPU waits (measured on B200: growing it for a merged
    // MSM pass's 3-6 GB round buffer held the scheduler 30-135 ms per
    // allocation, and a few in a row left the GPU idle for up to 3 s).  A
    // reservation that fails leaves the pool to grow on demand.
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
      const uint64_t margin = 4ull << 30;
      const uint64_t want = std::min<uint64_t>(adm_.budget(), free_b > margin ? free_b - margin : 0);
      if (want >= (1ull << 30)) reserve_pool(want, s_ntt_[0]);
    }
    // one pinned mailbox per stream slot; a slot is reused only after the
    // wave that used it retired (waves retire in launch order)
    // per job: an MSM slot, plus room for the multi-MSM offsets (one word)
    slot_words_ = 2 + (kMsmSlotWords + 1) * (uint64_t)max_wave_ + 2;
    ZK_TRY("cudaMallocHost(mailbox)", cudaMallocHost((void**)&mailbox_, kStreams * slot_words_ * 8));
    // the batch pass lists are uploaded from pinned memory: a copy from
    // pageable memory may make the enqueueing thread wait for the stream
    ZK_TRY("cudaMallocHost(pass stage)",
           cudaMallocHost((void**)&pass_stage_, kStreams * kPassStage * sizeof(BatchPass)));
    sched_ = std::thread([this] { sched_loop(); });
    comp_ = std::thread([this] { comp_loop(); });
    return ZKGPU_OK;
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_sched_.notify_all();
    cv_comp_.notify_all();
    if (sched_.joinable()) sched_.join();
    if (comp_.joinable()) comp_.join();
    cudaSetDevice(device_);
    cudaDeviceSynchronize();
    for (auto& b : bases_) cudaFree(b.d);
    if (mailbox_) cudaFreeHost(mailbox_);
    if (pass_stage_) cudaFreeHost(pass_stage_);
    // the reserved pool memory stays with the library for later calls (as
    // all pooled memory does); zkgpu_release_cached gives it back
    for (int i = 0; i < kStreams; i++) {
      if (s_ntt_[i]) cudaStreamDestroy(s_ntt_[i]);
      if (s_msm_[i]) cudaStreamDestroy(s_msm_[i]);
    }
  }

  int add_bases(const uint64_t* xy, uint64_t n, uint32_t* id) {
    const uint64_t bytes = n * 64;
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (!adm_.reserve(bytes)) return ZKGPU_EADMIT;
      peak_ = std::max(peak_, adm_.used() + adm_.reserved());
    }
    BaseSet b;
    b.n = n;
    // resident bases are kept in the curve arithmetic's R' form: converted
    // once here (in place) instead of on every MSM over them
    cudaError_t e = cudaSetDevice(device_);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b.d, std::max<uint64_t>(bytes, 64));
    if (e == cudaSuccess) e = cudaMemcpy(b.d, xy, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = msm_convert_bases(b.d, b.d, n, s_msm_[0]);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_msm_[0]);
    if (e != cudaSuccess) {
      if (b.d) cudaFree(b.d);
      std::lock_guard<std::mutex> lk(mu_);
      adm_.unreserve(bytes);
      return status_of("add_bases", e);
    }
    std::lock_guard<std::mutex> lk(mu_);
    bases_.push_back(b);
    *id = (uint32_t)bases_.size() - 1;
    return ZKGPU_OK;
  }

  int submit(const zkgpu_job* job, uint64_t* ticket) {
    auto rec = std::make_unique<JobRec>();
    rec->job = *job;
    rec->bytes = job->kind == ZKGPU_KIND_MSM ? msm_job_bytes(job->n, device_) : zkgpu_job_footprint(job);
    rec->t_submit = clk::now();
    std::lock_guard<std::mutex> lk(mu_);
    if (stop_) return ZKGPU_EBUSY;
    rec->ticket = next_ticket_++;
    submitted_++;
    if (job->kind == ZKGPU_KIND_MSM && (job->bases_id >= bases_.size() || job->n > bases_[job->bases_id].n)) {
      rejected_++;
      return ZKGPU_EINVAL;
    }
    if (!adm_.push(rec->ticket, rec->bytes)) {
      rejected_++;
      return ZKGPU_EADMIT;
    }
    *ticket = rec->ticket;
    jobs_.emplace(rec->ticket, std::move(rec));
    cv_sched_.notify_one();
    return ZKGPU_OK;
  }

  int wait(uint64_t ticket, uint32_t timeout_ms, double* latency_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) return ZKGPU_EINVAL;
    JobRec* r = it->second.get();
    auto done = [&] { return r->status >= 0; };
    if (timeout_ms == 0)
      cv_done_.wait(lk, done);
    else if (!cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
      return ZKGPU_ETIMEOUT;
    if (r->taken) return ZKGPU_EINVAL;  // already waited for
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    const int st = r->status;
    // a job can complete before its wave retires; the wave still reads the
    // record until then, so the retirement erases it
    if (r->retired)
      jobs_.erase(it);
    else
      r->taken = true;
    return st;
  }

  void stats(zkgpu_server_stats* o) {
    std::lock_guard<std::mutex> lk(mu_);
    o->submitted = submitted_;
    o->rejected = rejected_;
    o->completed = completed_;
    o->failed = failed_;
    o->waves = waves_;
    o->batch_launches = batch_launches_;
    o->hbm_budget = adm_.budget() + adm_.reserved();
    o->hbm_used = adm_.used() + adm_.reserved() + adm_.external();
    o->hbm_peak = peak_;
    o->pending = adm_.pending();
    o->inflight = inflight_jobs_;
    o->msm_merged_passes = merged_passes_;
    o->msm_merged_jobs = merged_jobs_;
    o->table_builds = table_cache_builds(device_) - builds0_;
    o->cache_clears = cache_clears_;
    o->memory_waits = memory_waits_;
    o->max_launch_us = max_launch_us_;
  }

 private:
  static constexpr int kStreams = 8;
  static constexpr int kEagerWaves = kStreams;
  // pass descriptors a stream slot's pinned upload buffer holds (a 64-job
  // wave of LDEs needs a few hundred)
  static constexpr size_t kPassStage = 2048;
  int eager_waves_ = kEagerWaves;
  // per MSM job in a wave's mailbox: window count, c, then the window sums
  static constexpr uint64_t kMsmSlotWords = 2 + 16 * (uint64_t)MSM_MAX_WINDOWS;

  void sched_loop() {
    cudaSetDevice(device_);
    int rr = 0;
    for (;;) {
      std::vector<JobRec*> batch;
      {
        std::unique_lock<std::mutex> lk(mu_);
        // Continuous batching: with fewer than kEagerWaves waves on the GPU a
        // wave starts with whatever is pending (low latency at low load);
        // with more in flight the GPU has queued work, so the next wave waits
        // until a full wave is pending or a wave retires (bigger waves, fewer
        // launches and better overlap under load).
        cv_sched_.wait(lk, [&] {
          return stop_ || (adm_.pending() > 0 && waves_inflight_ < kStreams &&
                           (waves_inflight_ < eager_waves_ || adm_.pending() >= max_wave_));
        });
        if (stop_) return;
        const uint64_t gen = retired_gen_;
        // the device's table caches count against the budget too
        adm_.set_external(table_cache_bytes(device_));
        for (uint64_t t : adm_.admit(max_wave_)) batch.push_back(jobs_.at(t).get());
        // the peak is what admitted work holds (tables other work cached
        // before anything was admitted are dropped below, not counted)
        if (!batch.empty()) peak_ = std::max(peak_, adm_.used() + adm_.reserved() + adm_.external());
        if (batch.empty()) {
          if (waves_inflight_ == 0 && adm_.external() > 0) {
            // nothing will retire to make room: drop the cached tables (work
            // still holding some keeps them alive) and try again
            cache_clears_++;
            lk.unlock();
            table_cache_clear(device_);
            continue;
          }
          // the head does not fit yet: wait until a wave retires and frees memory
          memory_waits_++;
          cv_sched_.wait(lk, [&] { return stop_ || retired_gen_ != gen; });
          continue;
        }
        inflight_jobs_ += batch.size();
        waves_inflight_++;
      }
      auto w = std::make_unique<Wave>();
      w->jobs = batch;
      w->s_ntt = s_ntt_[rr];
      w->s_msm = s_msm_[rr];
      w->mailbox = mailbox_ + rr * slot_words_;
      w->pass_stage = pass_stage_ + (size_t)rr * kPassStage;
      rr = (rr + 1) % kStreams;
      const auto tl0 = clk::now();
      launch_wave(*w);
      const uint64_t tl_us = (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(clk::now() - tl0).count();
      {
        std::lock_guard<std::mutex> lk(mu_);
        max_launch_us_ = std::max(max_launch_us_, tl_us);
        waves_++;
        inflight_.push_back(std::move(w));
      }
      cv_comp_.notify_one();
    }
  }

  // Enqueue one wave: allocations, uploads, one batch launch, MSMs, downloads.
  void launch_wave(Wave& w) {
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t x) {
      if (e == cudaSuccess && x != cudaSuccess) e = x;
      return e == cudaSuccess;
    };
    cudaEventCreateWithFlags(&w.ev_ntt, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&w.ev_msm, cudaEventDisableTiming);
    w.mailbox[0] = 0;
    uint64_t* next_msm_slot = w.mailbox + 2;
    struct NttItem {
      NttTablesRef t;
      fe* data;
      fe* tmp;
      PowTablesRef pre;
      host::Fr post;
      bool has_post;
      PowTablesRef post_tab;  // final pass: output i times table power i
      uint64_t nonzero;           // first pass: inputs past this are zero padding
      int level0;
      int dep_job;  // index in items of the transform this one follows, or -1
    };
    std::vector<NttItem> items;
    std::vector<std::pair<JobRec*, fe*>> ntt_outputs;  // device result -> job
    std::vector<void*> frees_ntt, frees_msm;
    // MSM jobs of this wave against the same resident bases run as one
    // multi-MSM pass (one sort and bucket pass, one launch sequence);
    // a lone MSM on its bases runs on its own
    std::map<uint32_t, std::vector<JobRec*>> msm_groups;
    for (JobRec* r : w.jobs)
      if (r->job.kind == ZKGPU_KIND_MSM) msm_groups[r->job.bases_id].push_back(r);
    // A group merges when its jobs fit one pass: 32-bit entry offsets (at
    // most 2^25 scalars) and the merged pass's device memory (one window
    // size from the mean job size, so a skewed group can need more than its
    // jobs alone) within the bytes the jobs were admitted with, plus what
    // the budget has free now (taken until the wave retires).
    std::map<uint32_t, bool> merge_ok;
    for (auto& g : msm_groups) {
      const std::vector<JobRec*>& grp = g.second;
      uint64_t tot = 0, max_n = 0, admitted = 0;
      for (const JobRec* r : grp) {
        tot += r->job.n;
        max_n = std::max<uint64_t>(max_n, r->job.n);
        admitted += r->bytes;
      }
      bool ok_merge = grp.size() >= 2 && tot <= (1ull << 25);
      if (ok_merge) {
        const uint64_t need = tot * 32 + grp.size() * (MSM_MAX_WINDOWS * 128ull + 4) +
                              msm_scratch_bytes(tot, (uint32_t)grp.size(), max_n, true, false, device_);
        if (need > admitted) {  // borrow the difference from the free budget until the wave retires
          std::lock_guard<std::mutex> lk(mu_);
          ok_merge = adm_.take(need - admitted);
          if (ok_merge) {
            w.extra_bytes += need - admitted;
            peak_ = std::max(peak_, adm_.used() + adm_.reserved() + adm_.external());
          }
        }
      }
      merge_ok[g.first] = ok_merge;
    }
    auto merged = [&](uint32_t bases_id) { return merge_ok[bases_id]; };
    for (auto& g : msm_groups) {
      std::vector<JobRec*>& grp = g.second;
      if (!merged(g.first)) continue;
      const BaseSet& bs = bases_[g.first];
      std::vector<uint32_t> off(grp.size() + 1, 0);
      uint64_t max_n = 0;
      for (size_t k = 0; k < grp.size(); k++) {
        off[k + 1] = off[k] + (uint32_t)grp[k]->job.n;
        max_n = std::max<uint64_t>(max_n, grp[k]->job.n);
      }
      const uint64_t n_total = off.back();
      fe *ds = nullptr, *dwin = nullptr;
      uint32_t* doff = nullptr;
      if (ok(zk::dmalloc((void**)&ds, std::max<uint64_t>(n_total, 1) * 32, w.s_msm)) &&
          ok(zk::dmalloc((void**)&dwin, grp.size() * MSM_MAX_WINDOWS * 128, w.s_msm)) &&
          ok(zk::dmalloc((void**)&doff, off.size() * 4, w.s_msm))) {
        // offsets travel through the wave's pinned mailbox tail so the copy
        // stays asynchronous
        uint32_t* h_off = reinterpret_cast<uint32_t*>(next_msm_slot);
        std::memcpy(h_off, off.data(), off.size() * 4);
        next_msm_slot += (off.size() * 4 + 7) / 8;
        ok(cudaMemcpyAsync(doff, h_off, off.size() * 4, cudaMemcpyHostToDevice, w.s_msm));
        for (size_t k = 0; k < grp.size(); k++)
          ok(cudaMemcpyAsync(ds + off[k], grp[k]->job.input, grp[k]->job.n * 32, cudaMemcpyHostToDevice,
                             w.s_msm));
        uint64_t nl = 0;
        MsmWindowsOut wo;
        wo.d_winsum = dwin;
        if (ok(msm_run_multi(ds, bs.d, doff, (uint32_t)grp.size(), n_total, max_n, w.s_msm, &nl, &wo, true))) {
          merged_passes_++;
          merged_jobs_ += grp.size();
          for (size_t k = 0; k < grp.size(); k++) {
            JobRec* r = grp[k];
            r->msm_out = next_msm_slot;
            next_msm_slot += kMsmSlotWords;
            r->msm_out[0] = wo.windows;
            r->msm_out[1] = wo.c;
            ok(cudaMemcpyAsync(r->msm_out + 2, dwin + (size_t)k * wo.windows * 4, wo.windows * 128ull,
                               cudaMemcpyDeviceToHost, w.s_msm));
          }
          for (JobRec* r : grp) record_done(r, w.s_msm);
        }
      }
      frees_msm.push_back(ds);
      frees_msm.push_back(dwin);
      frees_msm.push_back(doff);
    }
    for (JobRec* r : w.jobs) {
      const zkgpu_job& j = r->job;
      if (j.kind == ZKGPU_KIND_MSM && merged(j.bases_id)) continue;  // ran above
      if (j.kind == ZKGPU_KIND_MSM) {
        // the window sums come back to the mailbox; the completion thread
        // does the Horner step on the host (host::fq::msm_combine_windows)
        fe *ds = nullptr, *dwin = nullptr;
        const BaseSet& bs = bases_[j.bases_id];
        if (ok(zk::dmalloc((void**)&ds, std::max<uint64_t>(j.n, 1) * 32, w.s_msm)) &&
            ok(zk::dmalloc((void**)&dwin, MSM_MAX_WINDOWS * 128, w.s_msm)) &&
            ok(cudaMemcpyAsync(ds, j.input, j.n * 32, cudaMemcpyHostToDevice, w.s_msm))) {
          uint64_t nl = 0;
          MsmWindowsOut wo;
          wo.d_winsum = dwin;
          if (ok(msm_run(ds, bs.d, j.n, nullptr, w.s_msm, 0, &nl, &wo, true))) {
            r->msm_out = next_msm_slot;
            next_msm_slot += kMsmSlotWords;
            r->msm_out[0] = wo.windows;
            r->msm_out[1] = wo.c;
            ok(cudaMemcpyAsync(r->msm_out + 2, dwin, wo.windows * 128ull, cudaMemcpyDeviceToHost, w.s_msm));
            record_done(r, w.s_msm);
          }
        }
        frees_msm.push_back(ds);
        frees_msm.push_back(dwin);
        continue;
      }
      const bool lde = j.kind == ZKGPU_KIND_LDE;
      const uint32_t L = lde ? j.log_ext : j.log_n;
      const size_t N = (size_t)1 << L, n = (size_t)1 << j.log_n;
      fe *d = nullptr, *tmp = nullptr;
      if (!ok(zk::dmalloc((void**)&d, N * 32, w.s_ntt)) || !ok(zk::dmalloc((void**)&tmp, N * 32, w.s_ntt)))
        break;
      frees_ntt.push_back(d);
      frees_ntt.push_back(tmp);
      ok(cudaMemcpyAsync(d, j.input, n * 32, cudaMemcpyHostToDevice, w.s_ntt));
      cudaError_t te;
      if (!lde) {
        NttItem it{};
        it.t = ntt_tables_get(device_, fr_of(j.omega), (int)j.log_n, w.s_ntt, &te);
        if (!it.t) {
          ok(te);
          break;
        }
        if (j.flags & ZKGPU_JOB_COSET) it.pre = pow_tables_get(device_, fr_of(j.coset), (int)j.log_n, w.s_ntt, &te);
        if ((j.flags & ZKGPU_JOB_COSET) && !it.pre) {
          ok(te);
          break;
        }
        it.has_post = (j.flags & ZKGPU_JOB_SCALE) != 0;
        it.post = fr_of(j.scale);
        it.data = d;
        it.tmp = tmp;
        it.level0 = 0;
        it.dep_job = -1;
        items.push_back(it);
      } else {
        // ifft in place on the first n slots; its last pass applies n^-1 g^i,
        // and the extended NTT skips the zero padding (as zkgpu_lagrange_to_extended)
        NttItem a{}, b{};
        const host::Fr div = fr_of(j.scale);
        a.t = ntt_tables_get(device_, fr_of(j.omega), (int)j.log_n, w.s_ntt, &te);
        b.t = ntt_tables_get(device_, fr_of(j.omega_ext), (int)j.log_ext, w.s_ntt, &te);
        a.post_tab = pow_tables_get(device_, fr_of(j.coset), (int)j.log_n, w.s_ntt, &te, &div);
        if (!a.t || !b.t || !a.post_tab) {
          ok(te == cudaSuccess ? cudaErrorInvalidValue : te);
          break;
        }
        if (b.t->plan.npass > 1 && N > n && n % (1ull << (j.log_ext - b.t->plan.bits[0])) != 0)
          ok(cudaMemsetAsync(d + n, 0, (N - n) * 32, w.s_ntt));
        a.data = d;
        a.tmp = tmp;
        a.has_post = false;
        a.level0 = 0;
        a.dep_job = -1;
        b.data = d;
        b.tmp = tmp;
        b.has_post = false;
        b.nonzero = n;
        b.level0 = a.t->plan.npass;
        b.dep_job = (int)items.size();
        items.push_back(a);
        items.push_back(b);
      }
      ntt_outputs.push_back({r, d});
    }
    if (e == cudaSuccess && !items.empty()) {
      // level-ordered work list over all transforms of the wave
      int max_level = 0;
      for (auto& it : items) max_level = std::max(max_level, it.level0 + it.t->plan.npass);
      std::vector<int> last_pass(items.size(), -1);
      uint64_t tiles = 0;
      for (int lvl = 0; lvl < max_level; lvl++) {
        for (size_t i = 0; i < items.size(); i++) {
          const NttItem& it = items[i];
          const int k = lvl - it.level0;
          if (k < 0 || k >= it.t->plan.npass) continue;
          BatchPass bp{};
          NttFuse fu;
          fu.pre = it.pre.get();
          fu.post = it.has_post ? &it.post : nullptr;
          fu.post_tab = it.post_tab.get();
          fu.nonzero = it.nonzero;
          const uint64_t ncta = ntt_pass_params(*it.t, k, it.data, it.tmp, fu, &bp.p);
          bp.B = (uint32_t)it.t->plan.bits[k];
          bp.ntiles = (uint32_t)ncta;
          bp.tile_base = (uint32_t)tiles;
          int dep = k > 0 ? last_pass[i] : (it.dep_job >= 0 ? last_pass[it.dep_job] : -1);
          bp.dep = dep < 0 ? ~0u : (uint32_t)dep;
          bp.dep_tiles = dep < 0 ? 0u : w.passes[dep].ntiles;
          last_pass[i] = (int)w.passes.size();
          w.passes.push_back(bp);
          tiles += ncta;
        }
      }
      BatchPass* dp = nullptr;
      uint32_t* dc = nullptr;
      const size_t np = w.passes.size();
      if (ok(zk::dmalloc((void**)&dp, np * sizeof(BatchPass), w.s_ntt)) &&
          ok(zk::dmalloc((void**)&dc, (2 + np) * 4, w.s_ntt)) &&
          ok(upload_passes(w, dp, np)) &&
          ok(cudaMemsetAsync(dc, 0, (2 + np) * 4, w.s_ntt))) {
        ok(ntt_batch_launch(dp, (uint32_t)np, (uint32_t)tiles, dc, dc + 2, dc + 1, grid_, w.s_ntt));
        ok(cudaMemcpyAsync(w.mailbox, dc + 1, 4, cudaMemcpyDeviceToHost, w.s_ntt));
        batch_launches_++;
      }
      frees_ntt.push_back(dp);
      frees_ntt.push_back(dc);
      // results back smallest first, each job complete when its own copy is
      // (a small job does not wait for a large one's download)
      auto out_bytes = [](const JobRec* r) {
        const zkgpu_job& j = r->job;
        return ((size_t)1 << (j.kind == ZKGPU_KIND_LDE ? j.log_ext : j.log_n)) * 32;
      };
      std::stable_sort(ntt_outputs.begin(), ntt_outputs.end(),
                       [&](const std::pair<JobRec*, fe*>& x, const std::pair<JobRec*, fe*>& y) {
                         return out_bytes(x.first) < out_bytes(y.first);
                       });
      for (auto& o : ntt_outputs) {
        ok(cudaMemcpyAsync(o.first->job.output, o.second, out_bytes(o.first), cudaMemcpyDeviceToHost, w.s_ntt));
        record_done(o.first, w.s_ntt);
      }
    }
    for (const NttItem& it : items) {
      w.tables.push_back(it.t);
      if (it.pre) w.tables.push_back(it.pre);
      if (it.post_tab) w.tables.push_back(it.post_tab);
    }
    for (void* p : frees_ntt)
      if (p) cudaFreeAsync(p, w.s_ntt);
    for (void* p : frees_msm)
      if (p) cudaFreeAsync(p, w.s_msm);
    cudaEventRecord(w.ev_ntt, w.s_ntt);
    cudaEventRecord(w.ev_msm, w.s_msm);
    if (e != cudaSuccess) w.status = status_of("server wave", e);
  }

  // the wave's pass list to device memory, through the slot's pinned buffer
  // (reused only after the slot's previous wave retired, as the mailbox);
  // a list longer than the buffer goes from the wave's own copy
  static cudaError_t upload_passes(Wave& w, BatchPass* dp, size_t np) {
    const void* src = w.passes.data();
    if (np <= kPassStage) {
      std::memcpy(w.pass_stage, w.passes.data(), np * sizeof(BatchPass));
      src = w.pass_stage;
    }
    return cudaMemcpyAsync(dp, src, np * sizeof(BatchPass), cudaMemcpyHostToDevice, w.s_ntt);
  }

  // per-job completion event on the stream that produced the job's result
  static void record_done(JobRec* r, cudaStream_t s) {
    if (!r->done_ev && cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming) != cudaSuccess) {
      r->done_ev = nullptr;  // fall back to the wave's completion
      return;
    }
    cudaEventRecord(r->done_ev, s);
  }

  // finish one job on the host (MSM: Horner step into the caller's output)
  // and wake its waiter; the wave's memory is released when the wave retires
  void finish_job(JobRec* r, int st) {
    if (st == ZKGPU_OK && r->job.kind == ZKGPU_KIND_MSM && r->msm_out) {
      uint64_t out[12];
      host::fq::msm_combine_windows(r->msm_out + 2, (uint32_t)r->msm_out[0], (uint32_t)r->msm_out[1], out);
      std::memcpy(r->job.output, out, 96);
    }
    const auto now = clk::now();
    {
      std::lock_guard<std::mutex> lk(mu_);
      r->status = st;
      r->t_done = now;
      if (st == ZKGPU_OK)
        completed_++;
      else
        failed_++;
    }
    cv_done_.notify_all();
  }

  // Completion: jobs of every wave in flight finish one by one as their own
  // result copies land; waves retire in launch order once both their streams
  // are done, which releases their memory to the budget.
  void comp_loop() {
    cudaSetDevice(device_);
    for (;;) {
      std::vector<Wave*> live;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_comp_.wait(lk, [&] { return !inflight_.empty() || stop_; });
        if (inflight_.empty()) return;  // stop_ and nothing left
        for (auto& w : inflight_) live.push_back(w.get());  // only this thread pops: pointers stay valid
      }
      bool progressed = false;
      for (Wave* w : live) {
        if (w->status != ZKGPU_OK) continue;
        for (JobRec* r : w->jobs) {
          if (r->status >= 0 || !r->done_ev || r->early_failed) continue;
          const cudaError_t q = cudaEventQuery(r->done_ev);
          if (q == cudaErrorNotReady) continue;
          progressed = true;
          // an NTT / LDE result is good only if the batch kernel met every
          // wait: its error flag was copied before any of the wave's results
          if (q != cudaSuccess || (r->job.kind != ZKGPU_KIND_MSM && (uint32_t)w->mailbox[0])) {
            r->early_failed = true;  // reported when the wave retires
            continue;
          }
          finish_job(r, ZKGPU_OK);
        }
      }
      for (;;) {  // retire finished waves in order
        Wave* w;
        {
          std::lock_guard<std::mutex> lk(mu_);
          if (inflight_.empty()) break;
          w = inflight_.front().get();
        }
        const cudaError_t q1 = cudaEventQuery(w->ev_ntt), q2 = cudaEventQuery(w->ev_msm);
        if (q1 == cudaErrorNotReady || q2 == cudaErrorNotReady) break;
        retire(w, q1, q2);
        progressed = true;
      }
      if (!progressed) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_comp_.wait_for(lk, std::chrono::microseconds(50));
      }
    }
  }

  void retire(Wave* w, cudaError_t e1, cudaError_t e2) {
    int st = w->status;
    if (st == ZKGPU_OK && (e1 != cudaSuccess || e2 != cudaSuccess))
      st = status_of("server wave sync", e1 != cudaSuccess ? e1 : e2);
    if (st == ZKGPU_OK && (uint32_t)w->mailbox[0]) st = ZKGPU_ETIMEOUT;
    for (JobRec* r : w->jobs)
      if (r->status < 0) finish_job(r, st);
    for (JobRec* r : w->jobs)
      if (r->done_ev) {
        cudaEventDestroy(r->done_ev);
        r->done_ev = nullptr;
      }
    cudaEventDestroy(w->ev_ntt);
    cudaEventDestroy(w->ev_msm);
    std::unique_ptr<Wave> keep;  // destroyed after the lock: it releases table references
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (JobRec* r : w->jobs) {
        adm_.release(r->bytes);
        r->retired = true;
        if (r->taken) jobs_.erase(r->ticket);
      }
      adm_.release(w->extra_bytes);
      inflight_jobs_ -= w->jobs.size();
      waves_inflight_--;
      retired_gen_++;
      keep = std::move(inflight_.front());
      inflight_.pop_front();
    }
    cv_done_.notify_all();
    cv_sched_.notify_all();
  }

  int device_;
  AdmissionQueue adm_;
  uint32_t max_wave_;
  int grid_ = 0;
  cudaStream_t s_ntt_[kStreams] = {}, s_msm_[kStreams] = {};
  std::mutex mu_;
  std::condition_variable cv_sched_, cv_comp_, cv_done_;
  std::unordered_map<uint64_t, std::unique_ptr<JobRec>> jobs_;
  std::deque<std::unique_ptr<Wave>> inflight_;
  std::vector<BaseSet> bases_;
  std::thread sched_, comp_;
  bool stop_ = false;
  uint64_t next_ticket_ = 1, submitted_ = 0, rejected_ = 0, completed_ = 0, failed_ = 0, waves_ = 0;
  uint64_t batch_launches_ = 0, peak_ = 0, inflight_jobs_ = 0, retired_gen_ = 0;
  uint64_t cache_clears_ = 0, memory_waits_ = 0, max_launch_us_ = 0;
  uint64_t builds0_ = table_cache_builds(device_);  // the cache's count when this server started
  std::atomic<uint64_t> merged_passes_{0}, merged_jobs_{0};
  int waves_inflight_ = 0;
  uint64_t* mailbox_ = nullptr;
  BatchPass* pass_stage_ = nullptr;
  uint64_t slot_words_ = 0;
};

}  // namespace zk

extern "C" uint64_t zkgpu_job_footprint(const zkgpu_job* j) {
  if (!j) return 0;
  switch (j->kind) {
    case ZKGPU_KIND_NTT:
      return 2 * ((uint64_t)1 << j->log_n) * 32 + 4096;
    case ZKGPU_KIND_LDE:
      return 2 * ((uint64_t)1 << j->log_ext) * 32 + 4096;
    case ZKGPU_KIND_MSM: {
      int dev = 0;
      cudaGetDevice(&dev);
      return zk::msm_job_bytes(j->n, dev);
    }
    default:
      return 0;
  }
}

extern "C" uint64_t zkgpu_admission_simulate(uint64_t budget, const uint64_t* fp, uint32_t n, int32_t* rounds) {
  zk::AdmissionQueue q(budget);
  for (uint32_t i = 0; i < n; i++) {
    if (!q.push(i, fp[i])) rounds[i] = -1;
  }
  uint64_t peak = 0;
  int32_t round = 0;
  while (q.pending()) {
    std::vector<uint64_t> adm = q.admit();
    peak = std::max(peak, q.used());
    for (uint64_t t : adm) rounds[t] = round;
    for (uint64_t t : adm) q.release(fp[t]);  // each admitted job finishes this round
    round++;
  }
  return peak;
}

extern "C" int zkgpu_server_create(int device, uint64_t hbm_budget_bytes, uint32_t max_wave_jobs, void** server) {
  if (!server) return ZKGPU_EINVAL;
  cudaStream_t s;
  int st = zk::bind_device(device, &s);
  if (st) return st;
  auto srv = std::make_unique<zk::Server>(device, hbm_budget_bytes, max_wave_jobs);
  st = srv->start();
  if (st) return st;
  *server = srv.release();
  return ZKGPU_OK;
}

extern "C" int zkgpu_server_add_bases(void* server, const uint64_t* xy, uint64_t n, uint32_t* id) {
  if (!server || !id || (n && !xy)) return ZKGPU_EINVAL;
  return static_cast<zk::Server*>(server)->add_bases(xy, n, id);
}

extern "C" int zkgpu_server_submit(void* server, const zkgpu_job* job, uint64_t* ticket) {
  if (!server || !job || !ticket || !job->output) return ZKGPU_EINVAL;
  if (job->kind == ZKGPU_KIND_NTT || job->kind == ZKGPU_KIND_LDE) {
    if (!job->input || job->log_n < 3 || job->log_n > (uint32_t)zk::NTT_MAX_LOG) return ZKGPU_EINVAL;
    zk::host::Fr w = zk::fr_of(job->omega);
    if (!zk::host::is_canonical(w) || !zk::host::is_primitive_root(w, job->log_n)) return ZKGPU_EINVAL;
    if (job->kind == ZKGPU_KIND_LDE) {
      zk::host::Fr we = zk::fr_of(job->omega_ext);
      if (job->log_ext < job->log_n || job->log_ext > (uint32_t)zk::NTT_MAX_LOG || !zk::host::is_canonical(we) ||
          !zk::host::is_primitive_root(we, job->log_ext))
        return ZKGPU_EINVAL;
    }
  } else if (job->kind == ZKGPU_KIND_MSM) {
    if ((job->n && !job->input) || job->n >= (1ull << 31)) return ZKGPU_EINVAL;
  } else {
    return ZKGPU_EINVAL;
  }
  return static_cast<zk::Server*>(server)->submit(job, ticket);
}

extern "C" int zkgpu_server_wait(void* server, uint64_t ticket, uint32_t timeout_ms, double* latency_ms) {
  if (!server) return ZKGPU_EINVAL;
  return static_cast<zk::Server*>(server)->wait(ticket, timeout_ms, latency_ms);
}

extern "C" int zkgpu_server_stats_get(void* server, zkgpu_server_stats* out) {
  if (!server || !out) return ZKGPU_EINVAL;
  static_cast<zk::Server*>(server)->stats(out);
  return ZKGPU_OK;
}

extern "C" void zkgpu_server_destroy(void* server) { delete static_cast<zk::Server*>(server); }
