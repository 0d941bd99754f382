// admission.hpp — HBM-budget admission for the serving loop (host only).
//
// Replaces the reference's per-GPU MB counters (src/gpulock.rs:133-226,
// src/config.rs:97-123), which admitted a job while `mem_total > mem_used`
// without checking the new job's own size (gpulock.rs:174) and waited with
// blocking receives / 1 s sleeps.  Here every job carries its device
// footprint; jobs are admitted strictly in arrival order while they fit in
// the free budget (no overtaking, so a large job cannot starve), a job larger
// than the whole budget is rejected at submission, and freed memory admits
// the next jobs immediately.
#pragma once
#include <cstdint>
#include <deque>
#include <vector>

namespace zk {

class AdmissionQueue {
 public:
  explicit AdmissionQueue(uint64_t budget) : budget_(budget) {}

  // false (reject) if the job can never fit
  bool push(uint64_t ticket, uint64_t bytes) {
    if (bytes > budget_) return false;
    q_.push_back({ticket, bytes});
    return true;
  }
  // permanently take memory (resident bases) out of the budget jobs share;
  // false if it is not free now
  bool reserve(uint64_t bytes) {
    if (bytes > budget_ - used_) return false;
    budget_ -= bytes;
    reserved_ += bytes;
    return true;
  }
  // give back a reservation (resident bases that failed to load)
  void unreserve(uint64_t bytes) {
    bytes = bytes > reserved_ ? reserved_ : bytes;
    reserved_ -= bytes;
    budget_ += bytes;
  }
  uint64_t reserved() const { return reserved_; }
  // device memory held outside the jobs (the library's table caches), set
  // before each admission round; it counts against the same budget
  void set_external(uint64_t bytes) { external_ = bytes; }
  uint64_t external() const { return external_; }
  // take `bytes` more for work already admitted (e.g. a merged pass that
  // needs more than its jobs' footprints) if they are free now; give them
  // back with release()
  bool take(uint64_t bytes) {
    if (used_ + external_ > budget_ || bytes > budget_ - used_ - external_) return false;
    used_ += bytes;
    return true;
  }
  // admit jobs in FIFO order while the head fits; returns admitted tickets
  std::vector<uint64_t> admit(size_t max_jobs = SIZE_MAX) {
    std::vector<uint64_t> out;
    while (!q_.empty() && out.size() < max_jobs && used_ + external_ <= budget_ &&
           q_.front().bytes <= budget_ - used_ - external_) {
      used_ += q_.front().bytes;
      out.push_back(q_.front().ticket);
      q_.pop_front();
    }
    return out;
  }
  void release(uint64_t bytes) { used_ = bytes > used_ ? 0 : used_ - bytes; }
  uint64_t used() const { return used_; }
  uint64_t budget() const { return budget_; }
  size_t pending() const { return q_.size(); }

 private:
  struct Item {
    uint64_t ticket, bytes;
  };
  uint64_t budget_;
  uint64_t used_ = 0;
  uint64_t reserved_ = 0;
  uint64_t external_ = 0;
  std::deque<Item> q_;
};

}  // namespace zk
