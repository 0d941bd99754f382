// curve.cuh — BN254 G1 (y^2 = x^3 + 3 over Fq) on device, XYZZ coordinates.
//
// A point (X, Y, ZZ, ZZZ) represents x = X/ZZ, y = Y/ZZZ with ZZ^3 = ZZZ^2;
// the identity is ZZ = 0.  Formulas are the EFD's "xyzz" set for a = 0:
// dbl-2008-s-1 (6M + 3S), mdbl-2008-s-1, madd-2008-s (8M + 2S) and
// add-2008-s (12M + 2S), with the degenerate cases (P == Q -> doubling,
// P == -Q -> identity) handled explicitly, which the reference's Jacobian
// code gets wrong (cuda/curve.cuh:13-20, 170-179: its "identity" (0,0,R) is
// not recognised as zero afterwards).  Affine inputs use (0, 0) for the
// identity (cuda/bn256.h:15-20).  All arithmetic is canonical (values < q)
// because the equality tests need canonical representatives.
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

__device__ __forceinline__ void xyzz_set_inf(xyzz_t& p) {
  set_zero(p.x);
  set_zero(p.y);
  set_zero(p.zz);
  set_zero(p.zzz);
}
__device__ __forceinline__ bool xyzz_is_inf(const xyzz_t& p) { return is_zero(p.zz); }
__device__ __forceinline__ bool aff_is_inf(const aff_t& p) { return is_zero(p.x) && is_zero(p.y); }

__device__ __forceinline__ void xyzz_from_aff(xyzz_t& r, const aff_t& q) {
  if (aff_is_inf(q)) {
    xyzz_set_inf(r);
    return;
  }
  cpy(r.x, q.x);
  cpy(r.y, q.y);
  set_one<P_q>(r.zz);
  set_one<P_q>(r.zzz);
}

// r = 2p  (dbl-2008-s-1, a = 0).  The identity doubles to itself (ZZ stays 0).
__device__ __forceinline__ void xyzz_dbl(xyzz_t& r, const xyzz_t& p) {
  uint32_t U[8], V[8], W[8], S[8], M[8], t[8];
  dbl<P_q>(U, p.y);
  sqr<P_q>(V, U);
  mul<P_q>(W, U, V);
  mul<P_q>(S, p.x, V);
  sqr<P_q>(M, p.x);
  dbl<P_q>(t, M);
  add<P_q>(M, M, t);  // M = 3 X^2
  uint32_t X3[8], Y3[8];
  sqr<P_q>(X3, M);
  dbl<P_q>(t, S);
  sub<P_q>(X3, X3, t);
  sub<P_q>(t, S, X3);
  mul<P_q>(Y3, M, t);
  mul<P_q>(t, W, p.y);
  sub<P_q>(Y3, Y3, t);
  mul<P_q>(r.zz, V, p.zz);
  mul<P_q>(r.zzz, W, p.zzz);
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
  dbl<P_q>(U, q.y);
  sqr<P_q>(V, U);
  mul<P_q>(W, U, V);
  mul<P_q>(S, q.x, V);
  sqr<P_q>(M, q.x);
  dbl<P_q>(t, M);
  add<P_q>(M, M, t);
  sqr<P_q>(r.x, M);
  dbl<P_q>(t, S);
  sub<P_q>(r.x, r.x, t);
  sub<P_q>(t, S, r.x);
  mul<P_q>(r.y, M, t);
  mul<P_q>(t, W, q.y);
  sub<P_q>(r.y, r.y, t);
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
  mul<P_q>(U2, q.x, p.zz);
  mul<P_q>(S2, q.y, p.zzz);
  sub<P_q>(P, U2, p.x);
  sub<P_q>(R, S2, p.y);
  if (is_zero(P)) {
    if (is_zero(R))
      xyzz_mdbl(p, q);
    else
      xyzz_set_inf(p);
    return;
  }
  uint32_t PP[8], PPP[8], Q[8], t[8];
  sqr<P_q>(PP, P);
  mul<P_q>(PPP, P, PP);
  mul<P_q>(Q, p.x, PP);
  sqr<P_q>(t, R);
  sub<P_q>(t, t, PPP);
  uint32_t X3[8];
  dbl<P_q>(X3, Q);
  sub<P_q>(X3, t, X3);
  sub<P_q>(t, Q, X3);
  mul<P_q>(t, R, t);
  uint32_t u[8];
  mul<P_q>(u, p.y, PPP);
  sub<P_q>(p.y, t, u);
  cpy(p.x, X3);
  mul<P_q>(p.zz, p.zz, PP);
  mul<P_q>(p.zzz, p.zzz, PPP);
}

// p += q (both XYZZ), add-2008-s with all special cases
__device__ __forceinline__ void xyzz_add(xyzz_t& p, const xyzz_t& q) {
  if (xyzz_is_inf(q)) return;
  if (xyzz_is_inf(p)) {
    p = q;
    return;
  }
  uint32_t U1[8], U2[8], S1[8], S2[8], P[8], R[8];
  mul<P_q>(U1, p.x, q.zz);
  mul<P_q>(U2, q.x, p.zz);
  mul<P_q>(S1, p.y, q.zzz);
  mul<P_q>(S2, q.y, p.zzz);
  sub<P_q>(P, U2, U1);
  sub<P_q>(R, S2, S1);
  if (is_zero(P)) {
    if (is_zero(R))
      xyzz_dbl(p, p);
    else
      xyzz_set_inf(p);
    return;
  }
  uint32_t PP[8], PPP[8], Q[8], t[8], X3[8];
  sqr<P_q>(PP, P);
  mul<P_q>(PPP, P, PP);
  mul<P_q>(Q, U1, PP);
  sqr<P_q>(t, R);
  sub<P_q>(t, t, PPP);
  dbl<P_q>(X3, Q);
  sub<P_q>(X3, t, X3);
  sub<P_q>(t, Q, X3);
  mul<P_q>(t, R, t);
  mul<P_q>(S1, S1, PPP);
  sub<P_q>(p.y, t, S1);
  cpy(p.x, X3);
  mul<P_q>(p.zz, p.zz, q.zz);
  mul<P_q>(p.zz, p.zz, PP);
  mul<P_q>(p.zzz, p.zzz, q.zzz);
  mul<P_q>(p.zzz, p.zzz, PPP);
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

// XYZZ -> Jacobian without inversion: (X ZZ^2, Y ZZ^3, ZZZ)
__device__ __forceinline__ void xyzz_to_jacobian(uint32_t out[24], const xyzz_t& p) {
  if (xyzz_is_inf(p)) {
#pragma unroll
    for (int i = 0; i < 24; i++) out[i] = 0;
    return;
  }
  uint32_t zz2[8], zz3[8];
  sqr<P_q>(zz2, p.zz);
  mul<P_q>(zz3, zz2, p.zz);
  mul<P_q>(out, p.x, zz2);
  mul<P_q>(out + 8, p.y, zz3);
  cpy(out + 16, p.zzz);
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
