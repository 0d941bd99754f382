// fq_inv.cuh — Fq inversion by the binary extended Euclidean algorithm in a
// fixed number of branch-free steps, for the MSM's batch-affine rounds.
//
// A Fermat inversion a^(q-2) is ~330 dependent Montgomery products: about
// 0.18 ms of latency per inversion on the FP64 product, which sets a floor
// under every batch-affine round.  Stein's binary algorithm needs only
// additions, subtractions and shifts: with u = a, v = q, x1 = 1, x2 = 0 and
// the invariants x1 a = u, x2 a = v (mod q), v odd, one step does
//   if u is odd: (u, v, x1, x2) <- u < v ? (v - u, u, x2 - x1, x1)
//                                        : (u - v, v, x1 - x2, x2)
//   u <- u / 2,  x1 <- x1 / 2 mod q
// Each step at least halves u v < q^2 < 2^508, so after 508 steps u = 0 and
// v = gcd(a, q) = 1, x2 = a^-1.  Every step is the same instruction sequence
// (masks, no branches), so the threads of a warp inverting different values
// never diverge.  __host__ __device__: the host tests run the same code.
#pragma once
#include <cstdint>

namespace zk {

struct FqInvConst {
  static constexpr uint32_t Q[8] = {0xd87cfd47u, 0x3c208c16u, 0x6871ca8du, 0x97816a91u,
                                    0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
};

// r = a^-1 mod q for a canonical, nonzero a (plain integers, 8 x 32-bit
// little-endian limbs); r is canonical.  a = 0 gives r = 0.
__host__ __device__ inline void fq_inv_binary(uint32_t r[8], const uint32_t a[8]) {
  constexpr uint32_t Q0 = 0xd87cfd47u, Q1 = 0x3c208c16u, Q2 = 0x6871ca8du, Q3 = 0x97816a91u, Q4 = 0x8181585du,
                     Q5 = 0xb85045b6u, Q6 = 0xe131a029u, Q7 = 0x30644e72u;
  const uint32_t q[8] = {Q0, Q1, Q2, Q3, Q4, Q5, Q6, Q7};
  uint32_t u[8], v[8], x1[8], x2[8];
  for (int i = 0; i < 8; i++) {
    u[i] = a[i];
    v[i] = q[i];
    x1[i] = i == 0 ? 1u : 0u;
    x2[i] = 0u;
  }
  for (int step = 0; step < 508; step++) {
    const uint32_t odd = u[0] & 1u;
    // d = u - v; lt = u < v
    uint32_t d[8];
    uint64_t br = 0;
    for (int i = 0; i < 8; i++) {
      const uint64_t t = (uint64_t)u[i] - v[i] - br;
      d[i] = (uint32_t)t;
      br = (t >> 32) & 1u;
    }
    const uint32_t lt = (uint32_t)br;
    const uint32_t m_odd = 0u - odd, m_swap = 0u - (odd & lt), m_lt = 0u - lt;
    // |u - v|
    uint32_t ad[8];
    uint64_t c = lt;
    for (int i = 0; i < 8; i++) {
      const uint64_t t = (uint64_t)(d[i] ^ m_lt) + c;
      ad[i] = (uint32_t)t;
      c = t >> 32;
    }
    // x1 - x2 and x2 - x1 mod q
    uint32_t dx[8], rx[8];
    uint64_t b1 = 0, b2 = 0;
    for (int i = 0; i < 8; i++) {
      const uint64_t t1 = (uint64_t)x1[i] - x2[i] - b1;
      const uint64_t t2 = (uint64_t)x2[i] - x1[i] - b2;
      dx[i] = (uint32_t)t1;
      rx[i] = (uint32_t)t2;
      b1 = (t1 >> 32) & 1u;
      b2 = (t2 >> 32) & 1u;
    }
    const uint32_t mb1 = 0u - (uint32_t)b1, mb2 = 0u - (uint32_t)b2;
    uint64_t c1 = 0, c2 = 0;
    for (int i = 0; i < 8; i++) {
      const uint64_t t1 = (uint64_t)dx[i] + (q[i] & mb1) + c1;
      const uint64_t t2 = (uint64_t)rx[i] + (q[i] & mb2) + c2;
      dx[i] = (uint32_t)t1;
      rx[i] = (uint32_t)t2;
      c1 = t1 >> 32;
      c2 = t2 >> 32;
    }
    // new v, x2 (swap case) and the new u, x1 before halving
    uint32_t nu[8], nx[8];
    for (int i = 0; i < 8; i++) {
      const uint32_t vi = (u[i] & m_swap) | (v[i] & ~m_swap);
      const uint32_t x2i = (x1[i] & m_swap) | (x2[i] & ~m_swap);
      const uint32_t dxi = (rx[i] & m_lt) | (dx[i] & ~m_lt);
      nu[i] = (ad[i] & m_odd) | (u[i] & ~m_odd);
      nx[i] = (dxi & m_odd) | (x1[i] & ~m_odd);
      v[i] = vi;
      x2[i] = x2i;
    }
    // u <- u / 2 (u is even here); x1 <- x1 / 2 mod q
    const uint32_t m_xodd = 0u - (nx[0] & 1u);
    uint32_t hx[8];
    uint64_t cx = 0;
    for (int i = 0; i < 8; i++) {
      const uint64_t t = (uint64_t)nx[i] + (q[i] & m_xodd) + cx;  // x + q < 2^255: no carry out
      hx[i] = (uint32_t)t;
      cx = t >> 32;
    }
    for (int i = 0; i < 7; i++) {
      u[i] = (nu[i] >> 1) | (nu[i + 1] << 31);
      x1[i] = (hx[i] >> 1) | (hx[i + 1] << 31);
    }
    u[7] = nu[7] >> 1;
    x1[7] = hx[7] >> 1;
  }
  for (int i = 0; i < 8; i++) r[i] = x2[i];
}

}  // namespace zk
