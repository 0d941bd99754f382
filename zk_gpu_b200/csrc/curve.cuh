// curve.cuh — BN254 G1 (y^2 = x^3 + 3 over Fq) on device, XYZZ coordinates.
//
// A point (X, Y, ZZ, ZZZ) represents x = X/ZZ, y = Y/ZZZ with ZZ^3 = ZZZ^2;
// the identity is ZZ = 0.  Formulas are the EFD's "xyzz" set for a = 0:
// dbl-2008-s-1 (6M + 3S), mdbl-2008-s-1, madd-2008-s (8M + 2S) and
// add-2008-s (12M + 2S), with the degenerate cases (P == Q -> doubling,
// P == -Q -> identity) handled explicitly, which the reference's Jacobian
// code gets wrong (cuda/curve.cuh:13-20, 170-179: its "identity" (0,0,R) is
// not recognised as zero afterwards).  Affine inputs use (0, 0) for the
// identity (cuda/bn256.h:15-20).
//
// Arithmetic form: every coordinate is kept in the R' = 2^260 Montgomery
// form of the FP64 52-bit-limb product (mul_rp: R'-form x R'-form -> R'-form),
// lazily reduced in [0, 2q); values are made canonical only where they are
// compared with zero.  to_rprime / from_rprime convert from / to the
// R = 2^256 form used in memory by the API (bit-identical to halo2curves).
#pragma once
#include "field.cuh"

namespace zk {

using P_q = FqP;

struct xyzz_t {
  uint32_t x[8], y[8], zz[8], zzz[8];
};
struct aff_t {
  uint32_t x[8], y[8];
};

// ---- lazy R'-form Fq helpers --------------------------------------------
// ZK_MSM_CALL_PRODUCT: 0 = every product inlined; 1 = only the products of
// the batch-affine apply pass (qmul_c / qsqr_c) are calls of one out-of-line
// product (mul_rp_out); 2 (the default) = every qmul / qsqr is such a call.
// Measured on B200 with bit-identical outputs, MSM of 2^22 / 2^20 / 2^18 /
// 2^16 points: inlined 14.85 / 5.77 / 3.14 / 2.01 ms, apply pass only
// 14.8 / 5.8 / 3.1 / 2.0 ms, every product 14.42 / 5.32 / 2.75 / 1.82 ms:
// the XYZZ reduction and tail kernels, which inline a dozen or more products
// per thread, lose their spills (112 B -> 0 in the window kernel at 255
// registers) and their instruction-cache misses.
#ifndef ZK_MSM_CALL_PRODUCT
#define ZK_MSM_CALL_PRODUCT 2
#endif
__device__ __forceinline__ void qmul(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
#if ZK_MSM_CALL_PRODUCT >= 2
  mul_rp_out<P_q>(r, a, b);
#else
  mul_rp<P_q>(r, a, b);
#endif
}
__device__ __forceinline__ void qsqr(uint32_t r[8], const uint32_t a[8]) { qmul(r, a, a); }
__device__ __forceinline__ void qmul_c(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
#if ZK_MSM_CALL_PRODUCT >= 1
  mul_rp_out<P_q>(r, a, b);
#else
  mul_rp<P_q>(r, a, b);
#endif
}
__device__ __forceinline__ void qsqr_c(uint32_t r[8], const uint32_t a[8]) { qmul_c(r, a, a); }
__device__ __forceinline__ void qadd(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) { add_lazy<P_q>(r, a, b); }
__device__ __forceinline__ void qsub(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) { sub_lazy<P_q>(r, a, b); }
__device__ __forceinline__ void qdbl(uint32_t r[8], const uint32_t a[8]) { add_lazy<P_q>(r, a, a); }
__device__ __forceinline__ bool qzero(const uint32_t a[8]) {
  uint32_t c[8];
  reduce_once<P_q>(c, a);
  return is_zero(c);
}
// x (R form, x * 2^256) -> x * 2^260, canonical: multiply by 2^264 mod q
__device__ __forceinline__ void to_rprime(uint32_t r[8], const uint32_t a[8]) {
  const uint32_t k[8] = {0xfaec667au, 0xfbdb0f2au, 0x9626b0ffu, 0xad825aedu,
                         0x09e2a0fcu, 0x276f48b7u, 0xef86e357u, 0x0d791464u};
  mul_rp<P_q>(r, a, k);
  reduce_once<P_q>(r, r);
}
// x * 2^260 (lazy) -> x * 2^256, canonical: multiply by 2^256 mod q
__device__ __forceinline__ void from_rprime(uint32_t r[8], const uint32_t a[8]) {
  uint32_t one_r[8];
  set_one<P_q>(one_r);  // the integer 2^256 mod q
  mul_rp<P_q>(r, a, one_r);
  reduce_once<P_q>(r, r);
}

__device__ __forceinline__ void xyzz_set_inf(xyzz_t& p) {
  set_zero(p.x);
  set_zero(p.y);
  set_zero(p.zz);
  set_zero(p.zzz);
}
__device__ __forceinline__ bool xyzz_is_inf(const xyzz_t& p) { return qzero(p.zz); }
__device__ __forceinline__ bool aff_is_inf(const aff_t& p) { return is_zero(p.x) && is_zero(p.y); }

__device__ __forceinline__ void xyzz_from_aff(xyzz_t& r, const aff_t& q) {
  if (aff_is_inf(q)) {
    xyzz_set_inf(r);
    return;
  }
  cpy(r.x, q.x);
  cpy(r.y, q.y);
  set_one_rp<P_q>(r.zz);
  set_one_rp<P_q>(r.zzz);
}

// r = 2p  (dbl-2008-s-1, a = 0).  The identity doubles to itself (ZZ stays 0).
__device__ __forceinline__ void xyzz_dbl(xyzz_t& r, const xyzz_t& p) {
  uint32_t U[8], V[8], W[8], S[8], M[8], t[8];
  qdbl(U, p.y);
  qsqr(V, U);
  qmul(W, U, V);
  qmul(S, p.x, V);
  qsqr(M, p.x);
  qdbl(t, M);
  qadd(M, M, t);  // M = 3 X^2
  uint32_t X3[8], Y3[8];
  qsqr(X3, M);
  qdbl(t, S);
  qsub(X3, X3, t);
  qsub(t, S, X3);
  qmul(Y3, M, t);
  qmul(t, W, p.y);
  qsub(Y3, Y3, t);
  qmul(r.zz, V, p.zz);
  qmul(r.zzz, W, p.zzz);
  cpy(r.x, X3);
  cpy(r.y, Y3);
}

// r = 2q for an affine q (mdbl-2008-s-1)
__device__ __forceinline__ void xyzz_mdbl(xyzz_t& r, const aff_t& q) {
  if (aff_is_inf(q)) {
    xyzz_set_inf(r);
    return;
  }
  uint32_t U[8], V[8], W[8], S[8], M[8], t[8];
  qdbl(U, q.y);
  qsqr(V, U);
  qmul(W, U, V);
  qmul(S, q.x, V);
  qsqr(M, q.x);
  qdbl(t, M);
  qadd(M, M, t);
  qsqr(r.x, M);
  qdbl(t, S);
  qsub(r.x, r.x, t);
  qsub(t, S, r.x);
  qmul(r.y, M, t);
  qmul(t, W, q.y);
  qsub(r.y, r.y, t);
  cpy(r.zz, V);
  cpy(r.zzz, W);
}

// p += q (affine), madd-2008-s with all special cases
__device__ __forceinline__ void xyzz_madd(xyzz_t& p, const aff_t& q) {
  if (aff_is_inf(q)) return;
  if (xyzz_is_inf(p)) {
    xyzz_from_aff(p, q);
    return;
  }
  uint32_t U2[8], S2[8], P[8], R[8];
  qmul(U2, q.x, p.zz);
  qmul(S2, q.y, p.zzz);
  qsub(P, U2, p.x);
  qsub(R, S2, p.y);
  if (qzero(P)) {
    if (qzero(R))
      xyzz_mdbl(p, q);
    else
      xyzz_set_inf(p);
    return;
  }
  uint32_t PP[8], PPP[8], Q[8], t[8];
  qsqr(PP, P);
  qmul(PPP, P, PP);
  qmul(Q, p.x, PP);
  qsqr(t, R);
  qsub(t, t, PPP);
  uint32_t X3[8];
  qdbl(X3, Q);
  qsub(X3, t, X3);
  qsub(t, Q, X3);
  qmul(t, R, t);
  uint32_t u[8];
  qmul(u, p.y, PPP);
  qsub(p.y, t, u);
  cpy(p.x, X3);
  qmul(p.zz, p.zz, PP);
  qmul(p.zzz, p.zzz, PPP);
}

// p += q (both XYZZ), add-2008-s with all special cases
__device__ __forceinline__ void xyzz_add(xyzz_t& p, const xyzz_t& q) {
  if (xyzz_is_inf(q)) return;
  if (xyzz_is_inf(p)) {
    p = q;
    return;
  }
  uint32_t U1[8], U2[8], S1[8], S2[8], P[8], R[8];
  qmul(U1, p.x, q.zz);
  qmul(U2, q.x, p.zz);
  qmul(S1, p.y, q.zzz);
  qmul(S2, q.y, p.zzz);
  qsub(P, U2, U1);
  qsub(R, S2, S1);
  if (qzero(P)) {
    if (qzero(R))
      xyzz_dbl(p, p);
    else
      xyzz_set_inf(p);
    return;
  }
  uint32_t PP[8], PPP[8], Q[8], t[8], X3[8];
  qsqr(PP, P);
  qmul(PPP, P, PP);
  qmul(Q, U1, PP);
  qsqr(t, R);
  qsub(t, t, PPP);
  qdbl(X3, Q);
  qsub(X3, t, X3);
  qsub(t, Q, X3);
  qmul(t, R, t);
  qmul(S1, S1, PPP);
  qsub(p.y, t, S1);
  cpy(p.x, X3);
  qmul(p.zz, p.zz, q.zz);
  qmul(p.zz, p.zz, PP);
  qmul(p.zzz, p.zzz, q.zzz);
  qmul(p.zzz, p.zzz, PPP);
}

// p = k * p for a small non-negative k (double-and-add, k < 2^32)
__device__ __forceinline__ void xyzz_mul_small(xyzz_t& p, uint32_t k) {
  xyzz_t acc;
  xyzz_set_inf(acc);
  if (k == 0 || xyzz_is_inf(p)) {
    p = acc;
    return;
  }
  const int top = 31 - __clz(k);
  acc = p;
  for (int b = top - 1; b >= 0; b--) {
    xyzz_dbl(acc, acc);
    if ((k >> b) & 1) xyzz_add(acc, p);
  }
  p = acc;
}

// XYZZ (R' form) -> Jacobian (R form, canonical) without inversion:
// (X ZZ^2, Y ZZ^3, ZZZ) represents the same point.
__device__ __forceinline__ void xyzz_to_jacobian(uint32_t out[24], const xyzz_t& p) {
  if (xyzz_is_inf(p)) {
#pragma unroll
    for (int i = 0; i < 24; i++) out[i] = 0;
    return;
  }
  uint32_t zz2[8], zz3[8], t[8];
  qsqr(zz2, p.zz);
  qmul(zz3, zz2, p.zz);
  qmul(t, p.x, zz2);
  from_rprime(out, t);
  qmul(t, p.y, zz3);
  from_rprime(out + 8, t);
  from_rprime(out + 16, p.zzz);
}

__device__ __forceinline__ void ld_aff(aff_t& q, const fe* p) {
  ld_fe(q.x, p);
  ld_fe(q.y, p + 1);
}
__device__ __forceinline__ void ld_xyzz(xyzz_t& q, const fe* p) {
  ld_fe(q.x, p);
  ld_fe(q.y, p + 1);
  ld_fe(q.zz, p + 2);
  ld_fe(q.zzz, p + 3);
}
__device__ __forceinline__ void st_xyzz(fe* p, const xyzz_t& q) {
  st_fe(p, q.x);
  st_fe(p + 1, q.y);
  st_fe(p + 2, q.zz);
  st_fe(p + 3, q.zzz);
}

}  // namespace zk
