// ntt_tile.cuh — the device side of one NTT pass (a CTA tile of radix-2^B
// DIF columns with the twist or the final digit-reversed store), shared by
// the per-pass kernels, the persistent batch kernel and their launchers.
//
// The launchers of the wide passes (B = 7..11) live in their own translation
// unit, ntt_pass_wide.cu, which compiles in parallel with ntt.cu and can take
// its own ptxas options.  With inlined products, the three register rounds of
// a wide pass made ptxas -O3 spill about 1.3 KB per thread at 128 registers
// and -O1 was faster; with the out-of-line products below, -O3 spills
// 200-380 B and runs the radix-2^8 and 2^9 plans as fast as or faster than
// -O1, so every pass is built at -O3.
#pragma once
#include <cuda_runtime.h>

#include "field.cuh"
#include "ntt.cuh"

namespace zk {

using P_r = FrP;

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t swz(uint32_t e) { return e ^ ((e >> 3) & 31u); }

template <int LO>
__device__ __forceinline__ uint32_t ins3(uint32_t q, uint32_t r) {
  return (q & ((1u << LO) - 1u)) | (r << LO) | ((q >> LO) << (LO + 3));
}

__device__ __forceinline__ void ld_smem_fe(uint32_t r[8], const uint32_t* plane0, uint32_t plane_stride, uint32_t a) {
#pragma unroll
  for (int k = 0; k < 8; k++) r[k] = plane0[k * plane_stride + a];
}
// a twiddle stored pre-split as 5 planes of 52-bit limbs (doubles)
__device__ __forceinline__ void ld_smem_tw(double r[5], const double* plane0, uint32_t plane_stride, uint32_t a) {
#pragma unroll
  for (int k = 0; k < 5; k++) r[k] = plane0[k * plane_stride + a];
}
__device__ __forceinline__ void st_smem_fe(uint32_t* plane0, uint32_t plane_stride, uint32_t a, const uint32_t r[8]) {
#pragma unroll
  for (int k = 0; k < 8; k++) plane0[k * plane_stride + a] = r[k];
}

// The products of a pass.  With ZK_NTT_CALL_PRODUCT (the default) the
// butterfly products are calls of one out-of-line product, its operands and
// result passed by value so that they stay in registers: a radix-8 round then
// runs one product's code from the instruction cache instead of a fresh
// inlined copy per butterfly, whose cache misses held the fully unrolled
// rounds back.  The products outside the rounds (the twist, the coset
// pre-multiply, the output scale) are calls only in passes of width
// B >= ZK_NTT_CALL_EDGE_MIN_B: inlined they overlap their loads and run
// faster in the narrow passes, while in the wide ones the shorter code and
// lower register pressure win.  Measured on B200 with bit-identical
// results, against the build that inlined every product (bench, autotuned
// plans): forward NTT 2^24 4.72 -> 4.45 ms, LDE 2^24 -> 2^26 25.9 -> 24.7 ms,
// 512 batched jobs of 2^10..2^20 31.8 -> 28.2 ms, the same jobs one call
// each 94 -> 71 ms.
#ifndef ZK_NTT_CALL_PRODUCT
#define ZK_NTT_CALL_PRODUCT 1
#endif
#ifndef ZK_NTT_CALL_EDGE_MIN_B
#define ZK_NTT_CALL_EDGE_MIN_B 7
#endif
struct Tw5 { double d[5]; };
template <class P>
__device__ __noinline__ Fe8 mul_rp_pre_call(const Fe8 a, const Tw5 b) {
  Fe8 r;
  mul_rp_pre<P>(r.w, a.w, b.d);
  return r;
}
template <bool CALL = (ZK_NTT_CALL_PRODUCT != 0)>
__device__ __forceinline__ void ntt_mul(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
#if ZK_NTT_CALL_PRODUCT
  if constexpr (!CALL) {
    mul_rp<P_r>(r, a, b);
    return;
  }
  mul_rp_out<P_r>(r, a, b);
#else
  mul_rp<P_r>(r, a, b);
#endif
}
__device__ __forceinline__ void ntt_mul_pre(uint32_t r[8], const uint32_t a[8], const double w[5]) {
#if ZK_NTT_CALL_PRODUCT
  Fe8 av;
  Tw5 wv;
#pragma unroll
  for (int k = 0; k < 8; k++) av.w[k] = a[k];
#pragma unroll
  for (int k = 0; k < 5; k++) wv.d[k] = w[k];
  const Fe8 rv = mul_rp_pre_call<P_r>(av, wv);
#pragma unroll
  for (int k = 0; k < 8; k++) r[k] = rv.w[k];
#else
  mul_rp_pre<P_r>(r, a, w);
#endif
}

// One round: registers hold i(r) = ins3<LO>(q, r); perform the DIF stages
// with butterfly bits HI-1 .. LO.  tws: inner roots w_m^e (e < m/2), 5 planes.
template <int B, int LO, int HI>
__device__ __forceinline__ void ntt_round(uint32_t x[8][8], uint32_t q, const double* tws) {
  constexpr uint32_t HALF = 1u << (B - 1);
#pragma unroll
  for (int b = HI - 1; b >= LO; b--) {
    const int rb = b - LO;
#pragma unroll
    for (int r = 0; r < 8; r++) {
      if (r & (1 << rb)) continue;
      const int r2 = r | (1 << rb);
      uint32_t t[8];
      sub_lazy<P_r>(t, x[r], x[r2]);
      add_lazy<P_r>(x[r], x[r], x[r2]);
      if constexpr (LO == 0) {
        // exponent is a compile-time constant: (r mod 2^b) << (B-1-b)
        const uint32_t e = (uint32_t)(r & ((1 << b) - 1)) << (B - 1 - b);
        if (e == 0) {
#pragma unroll
          for (int k = 0; k < 8; k++) x[r2][k] = t[k];
        } else {
          double w[5];
          ld_smem_tw(w, tws, HALF, e);
          ntt_mul_pre(x[r2], t, w);
        }
      } else {
        const uint32_t e = ((q & ((1u << LO) - 1u)) | ((uint32_t)(r & ((1 << rb) - 1)) << LO)) << (B - 1 - b);
        double w[5];
        ld_smem_tw(w, tws, HALF, e);
        ntt_mul_pre(x[r2], t, w);
      }
    }
  }
}

template <int B, int LO_CUR, int LO_NEXT>
__device__ __forceinline__ void ntt_exchange(uint32_t x[8][8], uint32_t q, uint32_t gbase, uint32_t* sm,
                                             uint32_t plane_stride, bool active) {
  if (active) {
#pragma unroll
    for (int r = 0; r < 8; r++) st_smem_fe(sm, plane_stride, swz(gbase + ins3<LO_CUR>(q, r)), x[r]);
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int r = 0; r < 8; r++) ld_smem_fe(x[r], sm, plane_stride, swz(gbase + ins3<LO_NEXT>(q, r)));
  }
  __syncthreads();
}

template <int B, int HI>
__device__ __forceinline__ void ntt_rounds(uint32_t x[8][8], uint32_t q, uint32_t gbase, uint32_t* sm,
                                           uint32_t plane_stride, const double* tws, bool active) {
  constexpr int LO = HI - 3 > 0 ? HI - 3 : 0;
  ntt_round<B, LO, HI>(x, q, tws);
  if constexpr (LO > 0) {
    constexpr int LO_N = LO - 3 > 0 ? LO - 3 : 0;
    ntt_exchange<B, LO, LO_N>(x, q, gbase, sm, plane_stride, active);
    ntt_rounds<B, LO>(x, q, gbase, sm, plane_stride, tws, active);
  }
}


#ifndef ZK_NTT_MIN_BLOCKS
#define ZK_NTT_MIN_BLOCKS 2
#endif

// One CTA tile of one pass.  `tile` plays the role of the block index.  In
// BATCH mode the CTA may be wider than the tile (G * T threads are active,
// the rest only join the barriers) and data is read through L2 only, since
// other CTAs of the same launch produced it.
template <int B, bool BATCH>
__device__ __forceinline__ void ntt_pass_tile(const PassParams& p, uint64_t tile, uint32_t* smem) {
  constexpr uint32_t M = 1u << B;
  constexpr uint32_t T = M / 8;  // threads per column
  const uint32_t G = p.G;
  const uint32_t plane_stride = G * M;
  double* tws = reinterpret_cast<double*>(smem + 8 * plane_stride);  // 8-byte aligned: 32 G M bytes in

  const uint32_t tid = threadIdx.x;
  const uint32_t g = tid / T, q = tid % T;
  const bool active = !BATCH || g < G;

  for (uint32_t e = tid; e < M / 2; e += blockDim.x) {
    uint32_t w[8];
    double wl[5];
    ld_fe_nc(w, p.inner + e);
    split52(wl, w);  // stored pre-split: 5 limb planes
#pragma unroll
    for (int k = 0; k < 5; k++) tws[k * (M / 2) + e] = wl[k];
  }

  // element indices are < 2^28: 32-bit arithmetic, powers of two as shifts
  const uint32_t t32 = (uint32_t)tile;
  const uint32_t log_G = __ffs(G) - 1;
  const uint32_t J = 1u << p.log_J;
  uint32_t o, col = 0, base, stride;
  if (!p.is_final) {
    const uint32_t log_cpo = p.log_J - log_G;  // columns per outer block = J / G
    o = t32 >> log_cpo;
    col = ((t32 & ((1u << log_cpo) - 1u)) << log_G) + g;
    base = ((o << B) << p.log_J) + col;
    stride = J;
  } else {
    const uint32_t log_rest = p.log_O - p.log_m1;  // rest_count = O / m_1
    const uint32_t rest = t32 & ((1u << log_rest) - 1u);
    const uint32_t k1 = ((t32 >> log_rest) << log_G) + g;
    o = (k1 << log_rest) + rest;
    base = o << B;
    stride = 1;
  }

  uint32_t x[8][8];
  if (active) {
    const uint32_t rows = p.in_rows ? p.in_rows : M;  // rows past in_rows are zero padding
#pragma unroll
    for (int r = 0; r < 8; r++) {
      if (q + T * r >= rows)
        set_zero(x[r]);
      else if (BATCH)
        ld_fe_cg(x[r], p.in + (base + (q + T * r) * stride));
      else
        ld_fe(x[r], p.in + (base + (q + T * r) * stride));
    }
  } else {
#pragma unroll
    for (int r = 0; r < 8; r++) set_zero(x[r]);
  }

  if (p.pre_lo && active) {
    const uint32_t mask = (1u << p.pre_shift) - 1u;
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const uint32_t xi = base + (q + T * r) * stride;  // first pass: global input index
      uint32_t a[8], b[8];
      ld_fe_nc(a, p.pre_lo + (xi & mask));
      ld_fe_nc(b, p.pre_hi + (xi >> p.pre_shift));
      ntt_mul<(B >= ZK_NTT_CALL_EDGE_MIN_B)>(a, a, b);
      ntt_mul<(B >= ZK_NTT_CALL_EDGE_MIN_B)>(x[r], x[r], a);
    }
  }
  __syncthreads();

  ntt_rounds<B, B>(x, q, g * M, smem, plane_stride, tws, active);
  if (!active) return;

  // element r now holds output k = bitrev_B(8q + r)
  if (!p.is_final) {
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const uint32_t k = __brev(8 * q + r) >> (32 - B);
      uint32_t w[8];
      const uint32_t kj = (k << p.log_J) + col;
      ld_fe_nc(w, p.twist + kj);
      ntt_mul<(B >= ZK_NTT_CALL_EDGE_MIN_B)>(x[r], x[r], w);
      st_fe(p.out + (((o << B) << p.log_J) + kj), x[r]);
    }
  } else {
    // rev(o): o = k_1 * 2^(b_2+..) + ... + k_(p-1);  rev = k_1 + 2^b_1 k_2 + ...
    uint32_t rev = 0, rem = o;
    uint32_t low_bits = 0, total = 0;
#pragma unroll
    for (int t = 0; t < NTT_MAX_PASS; t++)
      if (t < (int)p.nprev) total += p.prev_bits[t];
    uint32_t above = total;
#pragma unroll
    for (int t = 0; t < NTT_MAX_PASS; t++) {
      if (t < (int)p.nprev) {
        above -= p.prev_bits[t];
        const uint32_t digit = rem >> above;
        rem &= (1u << above) - 1u;
        rev |= digit << low_bits;
        low_bits += p.prev_bits[t];
      }
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const uint32_t k = __brev(8 * q + r) >> (32 - B);
      uint32_t v[8];
      const uint32_t kout = rev + (k << total);  // natural output index
      if (p.post_lo) {
        uint32_t a[8], b[8];
        ld_fe_nc(a, p.post_lo + (kout & ((1u << p.post_shift) - 1u)));
        ld_fe_nc(b, p.post_hi + (kout >> p.post_shift));
        ntt_mul<(B >= ZK_NTT_CALL_EDGE_MIN_B)>(a, a, b);
        ntt_mul<(B >= ZK_NTT_CALL_EDGE_MIN_B)>(v, x[r], a);
        reduce_once<P_r>(v, v);
      } else if (p.has_post) {
        ntt_mul<(B >= ZK_NTT_CALL_EDGE_MIN_B)>(v, x[r], p.post.w);
        reduce_once<P_r>(v, v);
      } else {
        reduce_once<P_r>(v, x[r]);
      }
      st_fe(p.out + kout, v);
    }
  }
}

template <int B>
__global__ void __launch_bounds__(256, ZK_NTT_MIN_BLOCKS) ntt_pass_kernel(const PassParams p) {
  extern __shared__ __align__(16) uint32_t smem[];
  ntt_pass_tile<B, false>(p, blockIdx.x, smem);
}

template <int B>
inline cudaError_t launch_pass(const PassParams& pp, uint64_t ncta, cudaStream_t s) {
  constexpr uint32_t M = 1u << B;
  const uint32_t threads = pp.G * (M / 8);
  const size_t smem = (size_t)8 * pp.G * M * 4 + (size_t)(M / 2) * 40;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    cudaFuncSetAttribute(ntt_pass_kernel<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set[dev & 63] = true;
  }
  ntt_pass_kernel<B><<<(unsigned)ncta, threads, smem, s>>>(pp);
  return cudaGetLastError();
}

// B = 7..11 (ntt_pass_wide.cu)
cudaError_t launch_pass_wide(int B, const PassParams& pp, uint64_t ncta, cudaStream_t s);

}  // namespace zk
