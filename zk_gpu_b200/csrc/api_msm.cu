// api_msm.cu — C-ABI entry points for the G1 MSM (declared in include/zkgpu.h).
#include <cstring>

#include "host_field.hpp"
#include "msm.cuh"
#include "runtime.cuh"

using zk::fe;

namespace {

// Host buffers in, normalised Jacobian (12 u64) out.
int msm_host(int device, const uint64_t* scalars, const uint64_t* bases_xy, uint64_t n, uint64_t out[12]) {
  if (!out || (n && (!scalars || !bases_xy)) || n >= (1ull << 31)) return ZKGPU_EINVAL;
  if (n == 0) {
    std::memset(out, 0, 96);
    return ZKGPU_OK;
  }
  cudaStream_t s;
  int st = zk::bind_device(device, &s);
  if (st) return st;
  // the per-window sums come back to the host, which does the Horner step
  // (host::fq::msm_combine_windows) and the normalisation
  fe *ds = nullptr, *db = nullptr, *dwin = nullptr;
  uint64_t win[zk::MSM_MAX_WINDOWS * 16];
  cudaError_t e = zk::dmalloc((void**)&ds, n * 32, s);
  if (e == cudaSuccess) e = zk::dmalloc((void**)&db, n * 64, s);
  if (e == cudaSuccess) e = zk::dmalloc((void**)&dwin, zk::MSM_MAX_WINDOWS * 128, s);
  if (e == cudaSuccess) e = zk::h2d_copy(ds, scalars, n * 32, s);
  if (e == cudaSuccess) e = zk::h2d_copy(db, bases_xy, n * 64, s);
  uint64_t nl = 0;
  zk::MsmWindowsOut wo;
  wo.d_winsum = dwin;
  if (e == cudaSuccess) e = zk::msm_run(ds, db, n, nullptr, s, 0, &nl, &wo);
  zk::count_launches(nl);
  if (e == cudaSuccess && wo.windows > zk::MSM_MAX_WINDOWS) e = cudaErrorInvalidValue;
  if (e == cudaSuccess) e = zk::d2h_copy(win, dwin, wo.windows * 128ull, s);
  if (ds) cudaFreeAsync(ds, s);
  if (db) cudaFreeAsync(db, s);
  if (dwin) cudaFreeAsync(dwin, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return zk::status_of("msm", e);
  if (e2 != cudaSuccess) return zk::status_of("msm sync", e2);
  zk::host::fq::msm_combine_windows(win, wo.windows, wo.c, out);
  return ZKGPU_OK;
}

}  // namespace

extern "C" uint64_t parallel_msm_api(size_t device_id, const uint64_t* data, const GpuAffine* bases, uint64_t lenght,
                                     GpuProjective* acc) {
  if (!acc) return ZKGPU_EINVAL;
  uint64_t out[12];
  int st = msm_host((int)device_id, data, reinterpret_cast<const uint64_t*>(bases), lenght, out);
  if (st) return (uint64_t)st;
  std::memcpy(acc->x, out, 32);
  std::memcpy(acc->y, out + 4, 32);
  std::memcpy(acc->z, out + 8, 32);
  return ZKGPU_OK;
}

extern "C" int zkgpu_msm(int device, const uint64_t* scalars, const uint64_t* bases_xy, uint64_t n,
                         uint64_t out_xyz[12]) {
  return msm_host(device, scalars, bases_xy, n, out_xyz);
}

extern "C" int zkgpu_msm_dev(int device, const uint64_t* d_scalars, const uint64_t* d_bases_xy, uint64_t n,
                             uint64_t* d_out_xyz, void* stream) {
  if (!d_out_xyz || (n && (!d_scalars || !d_bases_xy)) || n >= (1ull << 31)) return ZKGPU_EINVAL;
  cudaStream_t own;
  int st = zk::bind_device(device, &own);
  if (st) return st;
  uint64_t nl = 0;
  cudaError_t e = zk::msm_run(reinterpret_cast<const fe*>(d_scalars), reinterpret_cast<const fe*>(d_bases_xy), n,
                              reinterpret_cast<fe*>(d_out_xyz), (cudaStream_t)stream, 0, &nl);
  zk::count_launches(nl);
  return zk::status_of("msm_dev", e);
}
