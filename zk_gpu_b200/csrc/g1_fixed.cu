// g1_fixed.cu — batch fixed-base scalar multiplication on G1: out_i = k_i * B
// in affine form, for many scalars k_i and one base point B.
//
// This is the generator of MSM bases (k_i * (1, 2) for seeded random k_i,
// the shape halo2's parameter setup produces), run on the device so a 2^22
// basis takes a fraction of a second instead of minutes of host time.
//
// Method: fixed 4-bit windows.  A table T[w][d] = d * 16^w * B (w < 64,
// 1 <= d < 16) is built once per call by 64 threads, normalised to affine;
// each scalar then costs at most 64 mixed additions (XYZZ madd) and one field
// inversion (Fermat, a^(q-2)) to return to affine.  All arithmetic is the
// R'-form product (mul_rp) of field.cuh; outputs are canonical R-form
// (Montgomery, 2^256) affine points, (0, 0) for the identity.
#include <cuda_runtime.h>

#include "curve.cuh"
#include "runtime.cuh"

namespace zk {
namespace {

// a^(q-2) = a^-1 for a != 0, R' form in and out (lazy in, canonical out)
__device__ void fq_inv_rp(uint32_t r[8], const uint32_t a[8]) {
  const uint32_t e[8] = {FqP::P0 - 2u, FqP::P1, FqP::P2, FqP::P3, FqP::P4, FqP::P5, FqP::P6, FqP::P7};
  uint32_t acc[8];
  set_one_rp<FqP>(acc);
  for (int w = 7; w >= 0; w--) {
    for (int b = 31; b >= 0; b--) {
      qsqr(acc, acc);
      if ((e[w] >> b) & 1u) qmul(acc, acc, a);
    }
  }
  reduce_once<FqP>(r, acc);
}

// XYZZ -> affine (R' form, canonical); identity -> (0, 0)
__device__ void xyzz_to_affine_rp(aff_t& o, const xyzz_t& p) {
  if (xyzz_is_inf(p)) {
    set_zero(o.x);
    set_zero(o.y);
    return;
  }
  uint32_t t[8], inv[8], izz[8], izzz[8];
  qmul(t, p.zz, p.zzz);
  fq_inv_rp(inv, t);       // 1 / (ZZ ZZZ)
  qmul(izz, inv, p.zzz);    // 1 / ZZ
  qmul(izzz, inv, p.zz);    // 1 / ZZZ
  qmul(o.x, p.x, izz);
  qmul(o.y, p.y, izzz);
  reduce_once<FqP>(o.x, o.x);
  reduce_once<FqP>(o.y, o.y);
}

// T[w * 16 + d] = d * 16^w * B (affine, R' form); T[w * 16] = (0, 0)
__global__ void g1_fixed_table_kernel(const fe* base, fe* table) {
  const int w = threadIdx.x;
  if (w >= 64) return;
  aff_t b;
  ld_aff(b, base);
  if (!aff_is_inf(b)) {
    to_rprime(b.x, b.x);
    to_rprime(b.y, b.y);
  }
  xyzz_t p, acc;
  xyzz_from_aff(p, b);
  for (int i = 0; i < 4 * w; i++) xyzz_dbl(p, p);
  aff_t o;
  set_zero(o.x);
  set_zero(o.y);
  st_fe(table + 2 * (w * 16), o.x);
  st_fe(table + 2 * (w * 16) + 1, o.y);
  acc = p;
  for (int d = 1; d < 16; d++) {
    xyzz_to_affine_rp(o, acc);
    st_fe(table + 2 * (w * 16 + d), o.x);
    st_fe(table + 2 * (w * 16 + d) + 1, o.y);
    xyzz_add(acc, p);
  }
}

__global__ void __launch_bounds__(128) g1_fixed_mul_kernel(const fe* scalars, uint64_t n, const fe* table,
                                                           fe* out) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t s[8];
  ld_fe(s, scalars + i);
  const uint32_t one[8] = {1, 0, 0, 0, 0, 0, 0, 0};
  mul<FrP>(s, s, one);  // canonical scalar
  xyzz_t acc;
  xyzz_set_inf(acc);
  for (int w = 0; w < 64; w++) {
    const uint32_t d = (s[w >> 3] >> (4 * (w & 7))) & 15u;
    if (d) {
      aff_t q;
      const fe* t = table + 2 * (w * 16 + d);
      ld_fe_nc(q.x, t);
      ld_fe_nc(q.y, t + 1);
      xyzz_madd(acc, q);
    }
  }
  aff_t o;
  xyzz_to_affine_rp(o, acc);
  if (!aff_is_inf(o)) {
    from_rprime(o.x, o.x);
    from_rprime(o.y, o.y);
  }
  st_fe(out + 2 * i, o.x);
  st_fe(out + 2 * i + 1, o.y);
}

}  // namespace
}  // namespace zk

using zk::fe;

extern "C" int zkgpu_g1_mul_fixed_dev(int device, const uint64_t base_xy[8], const uint64_t* d_scalars, uint64_t n,
                                      uint64_t* d_out_xy, void* stream) {
  if (!base_xy || (n && (!d_scalars || !d_out_xy)) || n >= (1ull << 31)) return ZKGPU_EINVAL;
  if (n == 0) return ZKGPU_OK;
  cudaStream_t own;
  int st = zk::bind_device(device, &own);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  fe *d_base = nullptr, *d_table = nullptr;
  cudaError_t e = zk::dmalloc((void**)&d_base, 64, s);
  if (e == cudaSuccess) e = zk::dmalloc((void**)&d_table, 64 * 16 * 64, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_base, base_xy, 64, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    zk::g1_fixed_table_kernel<<<1, 64, 0, s>>>(d_base, d_table);
    const uint64_t blocks = (n + 127) / 128;
    zk::g1_fixed_mul_kernel<<<(unsigned)blocks, 128, 0, s>>>(reinterpret_cast<const fe*>(d_scalars), n, d_table,
                                                              reinterpret_cast<fe*>(d_out_xy));
    e = cudaGetLastError();
    zk::count_launches(2);
  }
  if (d_base) cudaFreeAsync(d_base, s);
  if (d_table) cudaFreeAsync(d_table, s);
  // the host copy of base_xy must stay valid until the copy above has run
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return zk::status_of("g1_mul_fixed", e);
  return zk::status_of("g1_mul_fixed sync", e2);
}
