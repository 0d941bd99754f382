// api_msm.cu — C-ABI entry points for the G1 MSM (declared in include/zkgpu.h).
#include "runtime.cuh"

extern "C" uint64_t parallel_msm_api(size_t, const uint64_t*, const GpuAffine*, uint64_t, GpuProjective*) {
  return ZKGPU_EINVAL;
}
extern "C" int zkgpu_msm(int, const uint64_t*, const uint64_t*, uint64_t, uint64_t*) { return ZKGPU_EINVAL; }
extern "C" int zkgpu_msm_dev(int, const uint64_t*, const uint64_t*, uint64_t, uint64_t*, void*) { return ZKGPU_EINVAL; }
