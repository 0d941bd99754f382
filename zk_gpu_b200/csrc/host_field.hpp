// host_field.hpp — host-side Fr arithmetic for the library's own bookkeeping
// (root-of-unity checks, per-pass roots, LDE constants).  4 x u64 little
// endian Montgomery limbs, the layout of cuda/bn256.h:10-13.  Not on the hot
// path: a few hundred products per call at most.
#pragma once
#include <cstdint>
#include <cstring>

namespace zk {
namespace host {

struct Fr {
  uint64_t v[4];
};

static constexpr uint64_t R_P[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL,
                                    0x30644e72e131a029ULL};
static constexpr uint64_t R_INV = 0xc2e1f593efffffffULL;
static constexpr uint64_t R_ONE[4] = {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL,
                                      0x0e0a77c19a07df2fULL};
static constexpr uint64_t R_R2[4] = {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL,
                                     0x0216d0b17f4e44a5ULL};

inline bool geq(const uint64_t a[4], const uint64_t b[4]) {
  for (int i = 3; i >= 0; i--) {
    if (a[i] != b[i]) return a[i] > b[i];
  }
  return true;
}
inline void sub_p(uint64_t a[4]) {
  unsigned __int128 br = 0;
  for (int i = 0; i < 4; i++) {
    unsigned __int128 d = (unsigned __int128)a[i] - R_P[i] - (uint64_t)br;
    a[i] = (uint64_t)d;
    br = (d >> 64) & 1;
  }
}
inline bool is_canonical(const Fr& a) { return !geq(a.v, R_P); }

inline Fr mul(const Fr& a, const Fr& b) {
  uint64_t t[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    uint64_t c = 0;
    for (int j = 0; j < 4; j++) {
      unsigned __int128 s = (unsigned __int128)a.v[j] * b.v[i] + t[j] + c;
      t[j] = (uint64_t)s;
      c = (uint64_t)(s >> 64);
    }
    unsigned __int128 s = (unsigned __int128)t[4] + c;
    t[4] = (uint64_t)s;
    t[5] = (uint64_t)(s >> 64);
    uint64_t m = t[0] * R_INV;
    s = (unsigned __int128)m * R_P[0] + t[0];
    c = (uint64_t)(s >> 64);
    for (int j = 1; j < 4; j++) {
      s = (unsigned __int128)m * R_P[j] + t[j] + c;
      t[j - 1] = (uint64_t)s;
      c = (uint64_t)(s >> 64);
    }
    s = (unsigned __int128)t[4] + c;
    t[3] = (uint64_t)s;
    t[4] = t[5] + (uint64_t)(s >> 64);
  }
  Fr r;
  std::memcpy(r.v, t, sizeof(r.v));
  if (t[4] || geq(r.v, R_P)) sub_p(r.v);
  return r;
}
inline Fr one() {
  Fr r;
  std::memcpy(r.v, R_ONE, sizeof(r.v));
  return r;
}
inline Fr zero() {
  Fr r{{0, 0, 0, 0}};
  return r;
}
inline Fr from_u64(uint64_t x) {
  Fr c{{x, 0, 0, 0}}, r2;
  std::memcpy(r2.v, R_R2, sizeof(r2.v));
  return mul(c, r2);
}
inline bool eq(const Fr& a, const Fr& b) { return std::memcmp(a.v, b.v, sizeof(a.v)) == 0; }
inline Fr neg(const Fr& a) {
  if (!(a.v[0] | a.v[1] | a.v[2] | a.v[3])) return a;
  Fr r;
  unsigned __int128 br = 0;
  for (int i = 0; i < 4; i++) {
    unsigned __int128 d = (unsigned __int128)R_P[i] - a.v[i] - (uint64_t)br;
    r.v[i] = (uint64_t)d;
    br = (d >> 64) & 1;
  }
  return r;
}
inline Fr add(const Fr& a, const Fr& b) {  // canonical inputs
  Fr r;
  unsigned __int128 c = 0;
  for (int i = 0; i < 4; i++) {
    c += (unsigned __int128)a.v[i] + b.v[i];
    r.v[i] = (uint64_t)c;
    c >>= 64;
  }
  if (geq(r.v, R_P)) sub_p(r.v);  // p < 2^254: no carry out of the top limb
  return r;
}
inline Fr sub(const Fr& a, const Fr& b) { return add(a, neg(b)); }
inline Fr pow_u64(Fr a, uint64_t e) {
  Fr r = one();
  while (e) {
    if (e & 1) r = mul(r, a);
    e >>= 1;
    if (e) a = mul(a, a);
  }
  return r;
}
inline Fr pow_2k(Fr a, unsigned k) {  // a^(2^k)
  for (unsigned i = 0; i < k; i++) a = mul(a, a);
  return a;
}
inline Fr inv(const Fr& a) {  // Fermat: a^(r-2)
  uint64_t e[4];
  std::memcpy(e, R_P, sizeof(e));
  e[0] -= 2;
  Fr r = one();
  for (int i = 3; i >= 0; i--)
    for (int b = 63; b >= 0; b--) {
      r = mul(r, r);
      if ((e[i] >> b) & 1) r = mul(r, a);
    }
  return r;
}
// true iff w has multiplicative order exactly 2^log_n (w^(n/2) == -1)
inline bool is_primitive_root(const Fr& w, unsigned log_n) {
  if (log_n == 0) return eq(w, one());
  Fr h = pow_2k(w, log_n - 1);
  return eq(h, neg(one()));
}


// ---- Fq (base field), used for the MSM's final normalisation -------------
namespace fq {
static constexpr uint64_t P[4] = {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL,
                                  0x30644e72e131a029ULL};
static constexpr uint64_t INV = 0x87d20782e4866389ULL;
static constexpr uint64_t ONE[4] = {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL,
                                    0x0e0a77c19a07df2fULL};
struct E {
  uint64_t v[4];
};
inline bool geq_p(const uint64_t a[4]) {
  for (int i = 3; i >= 0; i--) {
    if (a[i] != P[i]) return a[i] > P[i];
  }
  return true;
}
inline void subp(uint64_t a[4]) {
  unsigned __int128 br = 0;
  for (int i = 0; i < 4; i++) {
    unsigned __int128 d = (unsigned __int128)a[i] - P[i] - (uint64_t)br;
    a[i] = (uint64_t)d;
    br = (d >> 64) & 1;
  }
}
inline E mul(const E& a, const E& b) {
  uint64_t t[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    uint64_t c = 0;
    for (int j = 0; j < 4; j++) {
      unsigned __int128 s = (unsigned __int128)a.v[j] * b.v[i] + t[j] + c;
      t[j] = (uint64_t)s;
      c = (uint64_t)(s >> 64);
    }
    unsigned __int128 s = (unsigned __int128)t[4] + c;
    t[4] = (uint64_t)s;
    t[5] = (uint64_t)(s >> 64);
    uint64_t m = t[0] * INV;
    s = (unsigned __int128)m * P[0] + t[0];
    c = (uint64_t)(s >> 64);
    for (int j = 1; j < 4; j++) {
      s = (unsigned __int128)m * P[j] + t[j] + c;
      t[j - 1] = (uint64_t)s;
      c = (uint64_t)(s >> 64);
    }
    s = (unsigned __int128)t[4] + c;
    t[3] = (uint64_t)s;
    t[4] = t[5] + (uint64_t)(s >> 64);
  }
  E r;
  std::memcpy(r.v, t, sizeof(r.v));
  if (t[4] || geq_p(r.v)) subp(r.v);
  return r;
}
inline E one() {
  E r;
  std::memcpy(r.v, ONE, sizeof(r.v));
  return r;
}
inline bool is_zero(const E& a) { return !(a.v[0] | a.v[1] | a.v[2] | a.v[3]); }
inline E inv(const E& a) {  // a^(q-2)
  uint64_t e[4];
  std::memcpy(e, P, sizeof(e));
  e[0] -= 2;
  E r = one();
  for (int i = 3; i >= 0; i--)
    for (int b = 63; b >= 0; b--) {
      r = mul(r, r);
      if ((e[i] >> b) & 1) r = mul(r, a);
    }
  return r;
}
// Jacobian (X, Y, Z) -> affine-normalised Jacobian (x, y, one); identity -> zeros
inline void normalize_jacobian(uint64_t xyz[12]) {
  E X, Y, Z;
  std::memcpy(X.v, xyz, 32);
  std::memcpy(Y.v, xyz + 4, 32);
  std::memcpy(Z.v, xyz + 8, 32);
  if (is_zero(Z)) {
    std::memset(xyz, 0, 96);
    return;
  }
  E zi = inv(Z), zi2 = mul(zi, zi), zi3 = mul(zi2, zi);
  E x = mul(X, zi2), y = mul(Y, zi3), o = one();
  std::memcpy(xyz, x.v, 32);
  std::memcpy(xyz + 4, y.v, 32);
  std::memcpy(xyz + 8, o.v, 32);
}
inline E add(const E& a, const E& b) {
  E r;
  unsigned __int128 c = 0;
  for (int i = 0; i < 4; i++) {
    c += (unsigned __int128)a.v[i] + b.v[i];
    r.v[i] = (uint64_t)c;
    c >>= 64;
  }
  if (c || geq_p(r.v)) subp(r.v);  // a, b < q: sum < 2q < 2^256 + q
  return r;
}
inline E sub(const E& a, const E& b) {
  E r;
  unsigned __int128 br = 0;
  for (int i = 0; i < 4; i++) {
    unsigned __int128 d = (unsigned __int128)a.v[i] - b.v[i] - (uint64_t)br;
    r.v[i] = (uint64_t)d;
    br = (d >> 64) & 1;
  }
  if (br) {  // add q back
    unsigned __int128 c = 0;
    for (int i = 0; i < 4; i++) {
      c += (unsigned __int128)r.v[i] + P[i];
      r.v[i] = (uint64_t)c;
      c >>= 64;
    }
  }
  return r;
}

// G1 points in XYZZ coordinates (x = X/ZZ, y = Y/ZZZ, identity ZZ = 0), R form,
// the host counterpart of curve.cuh's formulas (EFD dbl-2008-s-1 and
// add-2008-s for a = 0, with the P = Q and P = -Q cases).
struct Xyzz {
  E x, y, zz, zzz;
};
inline void xyzz_dbl(Xyzz& p) {
  if (is_zero(p.zz)) return;
  const E U = add(p.y, p.y), V = mul(U, U), W = mul(U, V), S = mul(p.x, V);
  const E X2 = mul(p.x, p.x), M = add(add(X2, X2), X2);
  const E X3 = sub(mul(M, M), add(S, S));
  const E Y3 = sub(mul(M, sub(S, X3)), mul(W, p.y));
  p.zz = mul(V, p.zz);
  p.zzz = mul(W, p.zzz);
  p.x = X3;
  p.y = Y3;
}
inline void xyzz_add(Xyzz& p, const Xyzz& q) {
  if (is_zero(q.zz)) return;
  if (is_zero(p.zz)) {
    p = q;
    return;
  }
  const E U1 = mul(p.x, q.zz), U2 = mul(q.x, p.zz), S1 = mul(p.y, q.zzz), S2 = mul(q.y, p.zzz);
  const E Pd = sub(U2, U1), R = sub(S2, S1);
  if (is_zero(Pd)) {
    if (is_zero(R))
      xyzz_dbl(p);
    else
      p.zz = p.zzz = E{{0, 0, 0, 0}};
    return;
  }
  const E PP = mul(Pd, Pd), PPP = mul(Pd, PP), Q = mul(U1, PP);
  const E X3 = sub(sub(mul(R, R), PPP), add(Q, Q));
  const E Y3 = sub(mul(R, sub(Q, X3)), mul(S1, PPP));
  p.zz = mul(mul(p.zz, q.zz), PP);
  p.zzz = mul(mul(p.zzz, q.zzz), PPP);
  p.x = X3;
  p.y = Y3;
}

// The last step of a windowed MSM on the host: Horner over the per-window
// sums, sum_w 2^(c w) S_w, then normalisation.  winsum holds `windows` XYZZ
// points (16 words each: X, Y, ZZ, ZZZ) in the device's R' = 2^260 form,
// lazily reduced (< 2q).  out: normalised Jacobian (x, y, one), zeros for the
// identity.  A single GPU thread needs ~1.5 ms for the ~250 dependent
// doublings; the host takes well under 0.1 ms.
inline void msm_combine_windows(const uint64_t* winsum, uint32_t windows, uint32_t c, uint64_t out[12]) {
  // R' -> R: times 2^252 mod q (mul divides by 2^256)
  static constexpr E K252 = {{0, 0, 0, 0x1000000000000000ULL}};  // 2^252 < q
  auto load = [&](uint32_t w) {
    Xyzz p;
    E* co[4] = {&p.x, &p.y, &p.zz, &p.zzz};
    for (int k = 0; k < 4; k++) {
      E v;
      std::memcpy(v.v, winsum + 16 * (size_t)w + 4 * k, 32);
      *co[k] = mul(v, K252);
    }
    return p;
  };
  Xyzz acc = windows ? load(windows - 1) : Xyzz{};
  for (int w = (int)windows - 2; w >= 0; w--) {
    for (uint32_t k = 0; k < c; k++) xyzz_dbl(acc);
    xyzz_add(acc, load((uint32_t)w));
  }
  if (!windows || is_zero(acc.zz)) {
    std::memset(out, 0, 96);
    return;
  }
  const E zz2 = mul(acc.zz, acc.zz), zz3 = mul(zz2, acc.zz);
  const E X = mul(acc.x, zz2), Y = mul(acc.y, zz3);
  std::memcpy(out, X.v, 32);
  std::memcpy(out + 4, Y.v, 32);
  std::memcpy(out + 8, acc.zzz.v, 32);
  normalize_jacobian(out);
}
}  // namespace fq

}  // namespace host
}  // namespace zk
