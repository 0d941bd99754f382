// fq_inv.cuh — Fq inversion by Bernstein–Yang divsteps in a fixed number of
// branch-free steps, for the MSM's batch-affine rounds.
//
// A Fermat inversion a^(q-2) is ~330 dependent Montgomery products (about
// 0.18 ms of latency on the FP64 product); Stein's binary algorithm needs
// ~500 steps of 256-bit subtractions, selects and shifts (~10^5
// instructions).  The divstep recurrence of D. J. Bernstein and B.-Y. Yang,
// "Fast constant-time gcd computation and modular inversion" (TCHES 2019),
//   delta > 0 and g odd: (delta, f, g) <- (1 - delta, g, (g - f) / 2)
//   g odd:               (delta, f, g) <- (1 + delta, f, (g + f) / 2)
//   g even:              (delta, f, g) <- (1 + delta, f, g / 2)
// starting from delta = 1, f = q (odd), g = a, reaches g = 0, f = +-1 after
// at most floor((49 d + 57) / 17) = 741 steps for d = 256-bit inputs
// (the paper's Theorem 11.2).  Each step looks only at the low bit of g,
// so 30 steps run on the low 32 bits of f and g alone and yield a 2x2
// integer matrix T with [f', g'] 2^30 = T [f, g]; the full-width numbers
// are updated once per 30 steps.  The cofactors d, e with f = d a and
// g = e a (mod q) follow the same matrix, divided by 2^30 modulo q
// (adding the multiple of q that clears the low 30 bits).  At the end
// a^-1 = f d (mod q).  25 batches (750 steps) and a bounded safety loop
// on g != 0; every step is the same instruction sequence (masks, no
// branches), so a warp's threads inverting different values never diverge.
//
// Numbers are signed radix-2^30 integers in 9 int32 limbs: limbs 0..7 in
// [0, 2^30), limb 8 signed, 270 bits.  |f|, |g| <= q < 2^254 throughout;
// |d|, |e| grow by less than q per batch (|u| + |v| <= 2^30 for the rows
// of T), so they stay below 30 q < 2^259 and every limb product plus
// carries fits an int64.  __host__ __device__: the host tests run the same
// code as the kernels.
#pragma once
#include <cstdint>

namespace zk {
namespace fqinv {

constexpr int32_t M30 = (1 << 30) - 1;
// limb i of q in radix 2^30 (a function: constant after unrolling, and
// usable in device code, unlike a namespace-scope array), and -q^-1 mod 2^30
__host__ __device__ constexpr int32_t QL(int i) {
  return i == 0 ? 0x187cfd47 : i == 1 ? 0x3082305b : i == 2 ? 0x071ca8d3 : i == 3 ? 0x205aa45a
       : i == 4 ? 0x01585d97 : i == 5 ? 0x0116da06 : i == 6 ? 0x1a029b85 : i == 7 ? 0x139cb84c : 0x3064;
}
constexpr uint32_t QNEG_INV30 = 0x24866389u;
constexpr int kBatches = 25;  // 750 divsteps >= 741

// 30 divsteps on the low 32 bits of f and g: returns the new delta and the
// matrix T = [[u, v], [q, r]] with (f', g') 2^30 = (u f + v g, q f + r g)
__host__ __device__ inline int32_t divsteps30(int32_t delta, uint32_t f, uint32_t g, int32_t t[4]) {
  uint32_t u = 1, v = 0, q = 0, r = 1;
#pragma unroll
  for (int i = 0; i < 30; i++) {
    const uint32_t godd = 0u - (g & 1u);
    const uint32_t pos = (uint32_t)((int32_t)(0 - delta) >> 31);  // all ones iff delta > 0
    const uint32_t sw = godd & pos;                               // the swapping case
    // swap: (f, g) <- (g, g - f); g odd: (f, g + f); g even: (f, g); then g / 2
    const uint32_t nf = (g & sw) | (f & ~sw), nu = (q & sw) | (u & ~sw), nv = (r & sw) | (v & ~sw);
    g += ((f ^ sw) - sw) & godd;
    q += ((u ^ sw) - sw) & godd;
    r += ((v ^ sw) - sw) & godd;
    f = nf;
    u = nu << 1;
    v = nv << 1;
    g >>= 1;
    delta = 1 + (int32_t)(((uint32_t)delta ^ sw) - sw);
  }
  t[0] = (int32_t)u;
  t[1] = (int32_t)v;
  t[2] = (int32_t)q;
  t[3] = (int32_t)r;
  return delta;
}

// (f, g) <- (u f + v g, q f + r g) / 2^30, exact
__host__ __device__ inline void update_fg(int32_t f[9], int32_t g[9], const int32_t t[4]) {
  const int64_t u = t[0], v = t[1], q = t[2], r = t[3];
  int64_t cf = u * f[0] + v * g[0], cg = q * f[0] + r * g[0];
  cf >>= 30;
  cg >>= 30;
#pragma unroll
  for (int i = 1; i < 9; i++) {
    cf += u * f[i] + v * g[i];
    cg += q * f[i] + r * g[i];
    f[i - 1] = (int32_t)(cf & M30);
    g[i - 1] = (int32_t)(cg & M30);
    cf >>= 30;
    cg >>= 30;
  }
  f[8] = (int32_t)cf;
  g[8] = (int32_t)cg;
}

// (d, e) <- (u d + v e, q d + r e) / 2^30 mod q: each row plus m q, with m
// in [0, 2^30) chosen to clear its low 30 bits, is then divided exactly
__host__ __device__ inline void update_de(int32_t d[9], int32_t e[9], const int32_t t[4]) {
  const int64_t u = t[0], v = t[1], q = t[2], r = t[3];
  const uint32_t sd = (uint32_t)t[0] * (uint32_t)d[0] + (uint32_t)t[1] * (uint32_t)e[0];
  const uint32_t se = (uint32_t)t[2] * (uint32_t)d[0] + (uint32_t)t[3] * (uint32_t)e[0];
  const int64_t md = (int64_t)((sd * QNEG_INV30) & (uint32_t)M30);
  const int64_t me = (int64_t)((se * QNEG_INV30) & (uint32_t)M30);
  int64_t cd = u * d[0] + v * e[0] + md * QL(0), ce = q * d[0] + r * e[0] + me * QL(0);
  cd >>= 30;
  ce >>= 30;
#pragma unroll
  for (int i = 1; i < 9; i++) {
    cd += u * d[i] + v * e[i] + md * QL(i);
    ce += q * d[i] + r * e[i] + me * QL(i);
    d[i - 1] = (int32_t)(cd & M30);
    e[i - 1] = (int32_t)(ce & M30);
    cd >>= 30;
    ce >>= 30;
  }
  d[8] = (int32_t)cd;
  e[8] = (int32_t)ce;
}

__host__ __device__ inline bool limbs_zero(const int32_t g[9]) {
  int32_t o = 0;
#pragma unroll
  for (int i = 0; i < 9; i++) o |= g[i];
  return o == 0;
}

}  // namespace fqinv

// r = a^-1 mod q for a canonical a (plain integers, 8 x 32-bit little-endian
// words); r is canonical.  a = 0 gives r = 0.
__host__ __device__ inline void fq_inv_divsteps(uint32_t r[8], const uint32_t a[8]) {
  using namespace fqinv;
  int32_t f[9], g[9], d[9], e[9];
#pragma unroll
  for (int i = 0; i < 9; i++) {
    f[i] = QL(i);
    d[i] = 0;
    e[i] = i == 0 ? 1 : 0;
    // bits [30 i, 30 i + 30) of a
    const int w = (30 * i) >> 5, b = (30 * i) & 31;
    uint64_t x = a[w];
    if (w + 1 < 8) x |= (uint64_t)a[w + 1] << 32;
    g[i] = (int32_t)((x >> b) & (uint64_t)M30);
  }
  int32_t delta = 1;
#pragma unroll 1
  for (int it = 0; it < kBatches + 4; it++) {
    if (it >= kBatches && limbs_zero(g)) break;  // the bound says g = 0 after kBatches
    int32_t t[4];
    delta = divsteps30(delta, (uint32_t)f[0] | ((uint32_t)f[1] << 30), (uint32_t)g[0] | ((uint32_t)g[1] << 30), t);
    update_de(d, e, t);
    update_fg(f, g, t);
  }
  // f = +-1 (limb 8 holds the sign): x = f d, then x + 32 q in (0, 64 q)
  const int64_t s = f[8] < 0 ? -1 : 1;
  int64_t c = 0;
  int32_t x[9];
#pragma unroll
  for (int i = 0; i < 9; i++) {
    c += s * d[i] + 32 * (int64_t)QL(i);
    x[i] = (int32_t)(c & M30);
    c >>= 30;
  }
  // radix 2^30 -> 9 words of 32 bits (the value is below 2^260)
  uint32_t w[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const int i = (32 * k) / 30, b = (32 * k) % 30;
    uint64_t v = (uint64_t)(uint32_t)x[i] >> b;
    if (i + 1 < 9) v |= (uint64_t)(uint32_t)x[i + 1] << (30 - b);
    if (i + 2 < 9) v |= (uint64_t)(uint32_t)x[i + 2] << (60 - b);
    w[k] = (uint32_t)v;
  }
  // subtract 32 q, 16 q, ..., q where it does not go negative: [0, q)
  constexpr uint32_t Q[8] = {0xd87cfd47u, 0x3c208c16u, 0x6871ca8du, 0x97816a91u,
                             0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
#pragma unroll
  for (int k = 5; k >= 0; k--) {
    uint32_t sh[9];
    sh[0] = Q[0] << k;
#pragma unroll
    for (int i = 1; i < 8; i++) sh[i] = k ? (Q[i] << k) | (Q[i - 1] >> (32 - k)) : Q[i];
    sh[8] = k ? Q[7] >> (32 - k) : 0u;
    uint32_t t[9];
    uint64_t br = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
      const uint64_t y = (uint64_t)w[i] - sh[i] - br;
      t[i] = (uint32_t)y;
      br = (y >> 63) & 1u;
    }
    const uint32_t keep = 0u - (uint32_t)br;  // all ones: w < k q, keep w
#pragma unroll
    for (int i = 0; i < 9; i++) w[i] = (w[i] & keep) | (t[i] & ~keep);
  }
#pragma unroll
  for (int i = 0; i < 8; i++) r[i] = w[i];
}

}  // namespace zk
