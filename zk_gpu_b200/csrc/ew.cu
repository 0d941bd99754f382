// ew.cu — element-wise Fr ops on device vectors of extended-domain
// evaluations, and the division by the vanishing polynomial on the coset
// (declared in include/zkgpu.h).
//
// halo2's quotient step works on polynomials in extended Lagrange form: it
// multiplies, adds and scales whole 2^log_ext vectors (custom gates, the
// permutation and lookup arguments, combined as h = h * y + e_i), then divides
// by t(X) = X^n - 1 evaluated on the coset and returns to coefficients
// (zkgpu_extended_to_coeff).  The reference offloads only the NTT and MSM;
// its one element-wise device op is distribute_powers (cuda/fft.cu:223-232).
//
// All of these are streaming passes: 64 or 32 B read and 32 B written per
// element, one or zero field products.  One product per element costs about
// 1/60 ns per element on the FP64-limb product against 96 B / 6.5 TB/s =
// 1/68 ns of HBM time, so the kernels are balanced close to the HBM roofline.
// Grids are a multiple of the SM count; each thread walks the vector with a
// grid stride, two elements per step so that four 16-B loads are in flight.
#include <cstring>

#include "field.cuh"
#include "host_field.hpp"
#include "prof.cuh"
#include "runtime.cuh"

namespace zk {
namespace {

using P_r = FrP;

// a * b * 2^-256 for canonical R-form a, b: the FP64 product gives
// a b 2^-260 (< 2p), four lazy doublings restore the factor 2^4.
__device__ __forceinline__ void mont_mul_data(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  mul_rp<P_r>(r, a, b);
#pragma unroll
  for (int k = 0; k < 4; k++) add_lazy<P_r>(r, r, r);
  reduce_once<P_r>(r, r);
}

template <int OP>
__device__ __forceinline__ void ew_one(fe* out, const fe* a, const fe* b, const fe& c_rp, uint64_t i) {
  uint32_t x[8], y[8], r[8];
  ld_fe(x, a + i);
  if (OP == ZKGPU_EW_MUL) {
    ld_fe(y, b + i);
    mont_mul_data(r, x, y);
  } else if (OP == ZKGPU_EW_ADD) {
    ld_fe(y, b + i);
    add<P_r>(r, x, y);
  } else if (OP == ZKGPU_EW_SUB) {
    ld_fe(y, b + i);
    sub<P_r>(r, x, y);
  } else if (OP == ZKGPU_EW_SCALE) {
    mul_rp<P_r>(r, x, c_rp.w);
    reduce_once<P_r>(r, r);
  } else {  // AXPY
    ld_fe(y, b + i);
    mul_rp<P_r>(r, x, c_rp.w);
    reduce_once<P_r>(r, r);
    add<P_r>(r, r, y);
  }
  st_fe(out + i, r);
}

template <int OP>
__global__ void __launch_bounds__(256) ew_kernel(fe* out, const fe* a, const fe* b, const fe c_rp, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  for (; i + stride < n; i += 2 * stride) {
    ew_one<OP>(out, a, b, c_rp, i);
    ew_one<OP>(out, a, b, c_rp, i + stride);
  }
  if (i < n) ew_one<OP>(out, a, b, c_rp, i);
}

constexpr int kMaxVanish = 64;  // distinct values of X^n - 1 on the coset (extension factor <= 64)
struct VanishInv {
  fe v[kMaxVanish];  // 1 / t_j in R' form
};

__global__ void __launch_bounds__(256) vanish_kernel(fe* d, const VanishInv tinv, uint32_t mask, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t x[8];
    ld_fe(x, d + i);
    mul_rp<P_r>(x, x, tinv.v[i & mask].w);
    reduce_once<P_r>(x, x);
    st_fe(d + i, x);
  }
}

fe to_fe_rp(const host::Fr& a) {
  const host::Fr r = host::mul(a, host::from_u64(16));
  fe out;
  std::memcpy(out.w, r.v, 32);
  return out;
}

unsigned stream_grid(uint64_t n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t want = (n + 511) / 512;  // two elements per thread per step at 256 threads
  const uint64_t cap = (uint64_t)sms * 8;
  return (unsigned)(want < cap ? (want ? want : 1) : cap);
}

}  // namespace
}  // namespace zk

using zk::fe;

extern "C" int zkgpu_ew_dev(int device, uint32_t op, uint64_t* d_out, const uint64_t* d_a, const uint64_t* d_b,
                            const uint64_t c[4], uint64_t n, void* stream) {
  if (op > ZKGPU_EW_AXPY) return ZKGPU_EINVAL;
  if (n == 0) return ZKGPU_OK;
  const bool needs_b = op != ZKGPU_EW_SCALE;
  const bool needs_c = op == ZKGPU_EW_SCALE || op == ZKGPU_EW_AXPY;
  if (!d_out || !d_a || (needs_b && !d_b) || (needs_c && !c)) return ZKGPU_EINVAL;
  fe c_rp{};
  if (needs_c) {
    zk::host::Fr cc;
    std::memcpy(cc.v, c, 32);
    if (!zk::host::is_canonical(cc)) return ZKGPU_EINVAL;
    c_rp = zk::to_fe_rp(cc);
  }
  cudaStream_t own;
  int st = zk::bind_device(device, &own);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  fe* out = reinterpret_cast<fe*>(d_out);
  const fe* a = reinterpret_cast<const fe*>(d_a);
  const fe* b = reinterpret_cast<const fe*>(d_b);
  const unsigned grid = zk::stream_grid(n);
  static const char* names[5] = {"ew_mul", "ew_add", "ew_sub", "ew_scale", "ew_axpy"};
  const double products = (op == ZKGPU_EW_ADD || op == ZKGPU_EW_SUB) ? 0.0 : (double)n;
  {
    zk::ProfScope ps(names[op], s, products, (double)n * (needs_b ? 96.0 : 64.0));
    switch (op) {
      case ZKGPU_EW_MUL: zk::ew_kernel<ZKGPU_EW_MUL><<<grid, 256, 0, s>>>(out, a, b, c_rp, n); break;
      case ZKGPU_EW_ADD: zk::ew_kernel<ZKGPU_EW_ADD><<<grid, 256, 0, s>>>(out, a, b, c_rp, n); break;
      case ZKGPU_EW_SUB: zk::ew_kernel<ZKGPU_EW_SUB><<<grid, 256, 0, s>>>(out, a, b, c_rp, n); break;
      case ZKGPU_EW_SCALE: zk::ew_kernel<ZKGPU_EW_SCALE><<<grid, 256, 0, s>>>(out, a, b, c_rp, n); break;
      default: zk::ew_kernel<ZKGPU_EW_AXPY><<<grid, 256, 0, s>>>(out, a, b, c_rp, n); break;
    }
  }
  zk::count_launches(1);
  return zk::status_of("zkgpu_ew_dev", cudaGetLastError());
}

extern "C" int zkgpu_divide_by_vanishing_dev(int device, uint64_t* d_ext, uint32_t log_n, uint32_t log_ext,
                                             const uint64_t g[4], const uint64_t omega_ext[4], void* stream) {
  namespace hf = zk::host;
  if (!d_ext || !g || !omega_ext) return ZKGPU_EINVAL;
  if (log_ext < log_n || log_ext > 28 || (1u << (log_ext - log_n)) > (uint32_t)zk::kMaxVanish) return ZKGPU_EINVAL;
  hf::Fr gg, we;
  std::memcpy(gg.v, g, 32);
  std::memcpy(we.v, omega_ext, 32);
  if (!hf::is_canonical(gg) || !hf::is_canonical(we) || !hf::is_primitive_root(we, log_ext)) return ZKGPU_EINVAL;
  // t_j = g^n w_ext^(n j) - 1 for j < 2^(log_ext - log_n), inverted on the host
  const uint32_t J = 1u << (log_ext - log_n);
  const hf::Fr step = hf::pow_2k(we, log_n);
  hf::Fr cur = hf::pow_2k(gg, log_n);
  zk::VanishInv tinv{};
  for (uint32_t j = 0; j < J; j++) {
    const hf::Fr t = hf::sub(cur, hf::one());
    if (hf::eq(t, hf::zero())) return ZKGPU_EINVAL;  // X^n - 1 vanishes on this coset
    tinv.v[j] = zk::to_fe_rp(hf::inv(t));
    cur = hf::mul(cur, step);
  }
  cudaStream_t own;
  int st = zk::bind_device(device, &own);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const uint64_t N = 1ull << log_ext;
  {
    zk::ProfScope ps("divide_by_vanishing", s, (double)N, (double)N * 64.0);
    zk::vanish_kernel<<<zk::stream_grid(N), 256, 0, s>>>(reinterpret_cast<fe*>(d_ext), tinv, J - 1, N);
  }
  zk::count_launches(1);
  return zk::status_of("zkgpu_divide_by_vanishing_dev", cudaGetLastError());
}
