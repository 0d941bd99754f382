// prof.cuh — opt-in CUDA-event timing of individual launches (diag.cu).
// A ProfScope placed around a launch records a start/stop event pair on the
// launch's stream when profiling is enabled (zkgpu_prof_enable), tagged with
// the kernel name and its algorithmic work (modmuls) and bytes.
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace zk {

class ProfScope {
 public:
  ProfScope(const char* name, cudaStream_t s, double work, double bytes);
  ~ProfScope();
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

 private:
  bool active_;
  cudaStream_t s_;
  std::string name_;
  double work_ = 0, bytes_ = 0;
  cudaEvent_t a_{}, b_{};
};

}  // namespace zk
