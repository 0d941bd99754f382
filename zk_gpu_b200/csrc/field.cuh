// field.cuh — BN254 Fr / Fq arithmetic for sm_100a on 8 x 32-bit limbs.
//
// Elements are 256-bit little-endian integers in Montgomery form with
// R = 2^256 — bit-identical to the reference's BigNum (cuda/bn256.h:10-13,
// 4 x u64 LE) and to halo2curves' Fr / Fq repr, so device buffers are the
// host buffers reinterpreted.  The moduli (cuda/bn256.h:37, :54) are both
// < 2^254, so 4p < R, which allows "lazy" forms:
//   mul_lazy : a, b < 2p  ->  a*b*R^-1 mod p  in [0, 2p)   (no final subtract)
//   add_lazy : a, b < 2p  ->  a + b           in [0, 2p)
//   sub_lazy : a, b < 2p  ->  a - b           in [0, 2p)
// and canonical forms (inputs < p, outputs < p) used where values are
// compared.  Every carry chain lives inside ONE asm statement: the carry
// flag is never assumed to survive between statements (the reference's
// gpu_math.h:31-77 macros rely on that; this file does not).
//
// Montgomery multiplication is CIOS over 32-bit words; each iteration adds
// a*b_i (lo then hi partial products, two madc chains), computes
// m = T0 * (-p^-1 mod 2^32) and adds m*p the same way, then drops T0.
// Cost: 8 x (33 IMAD + 2 IADD) per product, all on the integer pipes.
#pragma once
#include <cstdint>

namespace zk {

struct fe {
  uint32_t w[8];
};

// ---- moduli (cuda/bn256.h:37-56) ----------------------------------------
struct FrP {
  static constexpr uint32_t P0 = 0xf0000001u, P1 = 0x43e1f593u, P2 = 0x79b97091u, P3 = 0x2833e848u,
                            P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t INV = 0xefffffffu;  // -p^-1 mod 2^32
  // R mod p (Montgomery one)
  static constexpr uint32_t O0 = 0x4ffffffbu, O1 = 0xac96341cu, O2 = 0x9f60cd29u, O3 = 0x36fc7695u,
                            O4 = 0x7879462eu, O5 = 0x666ea36fu, O6 = 0x9a07df2fu, O7 = 0x0e0a77c1u;
  // 2^261 mod p (the one of the 2^261 form of the IMAD product mul_r29)
  static constexpr uint32_t Q0 = 0x8fffff57u, Q1 = 0x2fd4e156u, Q2 = 0xa494b01au, Q3 = 0x75bba827u,
                            Q4 = 0x819caa80u, Q5 = 0x5301fa84u, Q6 = 0x563d4475u, Q7 = 0x0dc83629u;
  // 2^260 mod p (the one of the R' = 2^260 form used by mul_rp)
  static constexpr uint32_t D0 = 0x3fffffacu, D1 = 0xb9db6b75u, D2 = 0x0f271055u, D3 = 0xcef7c838u,
                            D4 = 0x818f016eu, D5 = 0x85a9201du, D6 = 0x1bb7724fu, D7 = 0x1f16424eu;
};
struct FqP {
  static constexpr uint32_t P0 = 0xd87cfd47u, P1 = 0x3c208c16u, P2 = 0x6871ca8du, P3 = 0x97816a91u,
                            P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t INV = 0xe4866389u;
  static constexpr uint32_t O0 = 0xc58f0d9du, O1 = 0xd35d438du, O2 = 0xf5c70b3du, O3 = 0x0a78eb28u,
                            O4 = 0x7879462cu, O5 = 0x666ea36fu, O6 = 0x9a07df2fu, O7 = 0x0e0a77c1u;
  static constexpr uint32_t Q0 = 0x157ccc21u, Q1 = 0x4e8384ebu, Q2 = 0x0ce148c3u, Q3 = 0xfb90a602u,
                            Q4 = 0x819caa36u, Q5 = 0x5301fa84u, Q6 = 0x563d4475u, Q7 = 0x0dc83629u;
  static constexpr uint32_t D0 = 0xf6fce4b4u, D1 = 0x45520880u, D2 = 0xbaa989a8u, D3 = 0x49890849u,
                            D4 = 0x818f014au, D5 = 0x85a9201du, D6 = 0x1bb7724fu, D7 = 0x1f16424eu;
};

#define ZK_P_OPS(P) "n"(P::INV), "n"(P::P0), "n"(P::P1), "n"(P::P2), "n"(P::P3), "n"(P::P4), "n"(P::P5), "n"(P::P6), "n"(P::P7)

// One CIOS iteration: T += a * b ; m = T0*inv ; T += m*p  (T is 9 words).
// Operands: %0-%8 T, %9-%16 a, %17 b, %18 inv, %19-%26 p.
#define ZK_CIOS_BODY                               \
  "{\n\t.reg .u32 m;\n\t"                          \
  "mad.lo.cc.u32  %0, %9, %17, %0;\n\t"            \
  "madc.lo.cc.u32 %1, %10, %17, %1;\n\t"           \
  "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"           \
  "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"           \
  "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"           \
  "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"           \
  "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"           \
  "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"           \
  "addc.u32       %8, %8, 0;\n\t"                  \
  "mad.hi.cc.u32  %1, %9, %17, %1;\n\t"            \
  "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"           \
  "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"           \
  "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"           \
  "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"           \
  "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"           \
  "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"           \
  "madc.hi.u32    %8, %16, %17, %8;\n\t"           \
  "mul.lo.u32     m, %0, %18;\n\t"                 \
  "mad.lo.cc.u32  %0, m, %19, %0;\n\t"             \
  "madc.lo.cc.u32 %1, m, %20, %1;\n\t"             \
  "madc.lo.cc.u32 %2, m, %21, %2;\n\t"             \
  "madc.lo.cc.u32 %3, m, %22, %3;\n\t"             \
  "madc.lo.cc.u32 %4, m, %23, %4;\n\t"             \
  "madc.lo.cc.u32 %5, m, %24, %5;\n\t"             \
  "madc.lo.cc.u32 %6, m, %25, %6;\n\t"             \
  "madc.lo.cc.u32 %7, m, %26, %7;\n\t"             \
  "addc.u32       %8, %8, 0;\n\t"                  \
  "mad.hi.cc.u32  %1, m, %19, %1;\n\t"             \
  "madc.hi.cc.u32 %2, m, %20, %2;\n\t"             \
  "madc.hi.cc.u32 %3, m, %21, %3;\n\t"             \
  "madc.hi.cc.u32 %4, m, %22, %4;\n\t"             \
  "madc.hi.cc.u32 %5, m, %23, %5;\n\t"             \
  "madc.hi.cc.u32 %6, m, %24, %6;\n\t"             \
  "madc.hi.cc.u32 %7, m, %25, %7;\n\t"             \
  "madc.hi.u32    %8, m, %26, %8;\n\t"             \
  "}"

// First iteration: T = a * b0 (T starts at zero), then the reduction step.
#define ZK_CIOS_FIRST                              \
  "{\n\t.reg .u32 m;\n\t"                          \
  "mul.lo.u32     %0, %9, %17;\n\t"                \
  "mul.lo.u32     %1, %10, %17;\n\t"               \
  "mul.lo.u32     %2, %11, %17;\n\t"               \
  "mul.lo.u32     %3, %12, %17;\n\t"               \
  "mul.lo.u32     %4, %13, %17;\n\t"               \
  "mul.lo.u32     %5, %14, %17;\n\t"               \
  "mul.lo.u32     %6, %15, %17;\n\t"               \
  "mul.lo.u32     %7, %16, %17;\n\t"               \
  "mad.hi.cc.u32  %1, %9, %17, %1;\n\t"            \
  "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"           \
  "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"           \
  "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"           \
  "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"           \
  "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"           \
  "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"           \
  "madc.hi.u32    %8, %16, %17, 0;\n\t"            \
  "mul.lo.u32     m, %0, %18;\n\t"                 \
  "mad.lo.cc.u32  %0, m, %19, %0;\n\t"             \
  "madc.lo.cc.u32 %1, m, %20, %1;\n\t"             \
  "madc.lo.cc.u32 %2, m, %21, %2;\n\t"             \
  "madc.lo.cc.u32 %3, m, %22, %3;\n\t"             \
  "madc.lo.cc.u32 %4, m, %23, %4;\n\t"             \
  "madc.lo.cc.u32 %5, m, %24, %5;\n\t"             \
  "madc.lo.cc.u32 %6, m, %25, %6;\n\t"             \
  "madc.lo.cc.u32 %7, m, %26, %7;\n\t"             \
  "addc.u32       %8, %8, 0;\n\t"                  \
  "mad.hi.cc.u32  %1, m, %19, %1;\n\t"             \
  "madc.hi.cc.u32 %2, m, %20, %2;\n\t"             \
  "madc.hi.cc.u32 %3, m, %21, %3;\n\t"             \
  "madc.hi.cc.u32 %4, m, %22, %4;\n\t"             \
  "madc.hi.cc.u32 %5, m, %23, %5;\n\t"             \
  "madc.hi.cc.u32 %6, m, %24, %6;\n\t"             \
  "madc.hi.cc.u32 %7, m, %25, %7;\n\t"             \
  "madc.hi.u32    %8, m, %26, %8;\n\t"             \
  "}"

#define ZK_T_OPS(T) "+r"(T[0]), "+r"(T[1]), "+r"(T[2]), "+r"(T[3]), "+r"(T[4]), "+r"(T[5]), "+r"(T[6]), "+r"(T[7]), "+r"(T[8])
#define ZK_A_OPS(a) "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7])

// r = a*b*R^-1 mod p, for a, b < 2p: result < 2p.
template <class P>
__device__ __forceinline__ void mul_lazy(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  uint32_t T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  asm(ZK_CIOS_FIRST : ZK_T_OPS(T) : ZK_A_OPS(a), "r"(b[0]), ZK_P_OPS(P));
#pragma unroll
  for (int i = 1; i < 8; i++) {
    // shift: drop T0 (zero), T8 becomes the new top, new T8 = 0
#pragma unroll
    for (int j = 0; j < 8; j++) T[j] = T[j + 1];
    T[8] = 0;
    asm(ZK_CIOS_BODY : ZK_T_OPS(T) : ZK_A_OPS(a), "r"(b[i]), ZK_P_OPS(P));
  }
#pragma unroll
  for (int j = 0; j < 8; j++) r[j] = T[j + 1];
}

// r = a + b - 2p if that does not borrow, else a + b.  Inputs < 2p.
template <class P>
__device__ __forceinline__ void add_lazy(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  uint32_t s[8], t[8], borrow;
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7])
      : ZK_A_OPS(a), ZK_A_OPS(b));
  // t = s - 2p
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7]), "=r"(borrow)
      : ZK_A_OPS(s), "n"((uint32_t)(P::P0 << 1)), "n"((P::P1 << 1) | (P::P0 >> 31)), "n"((P::P2 << 1) | (P::P1 >> 31)),
        "n"((P::P3 << 1) | (P::P2 >> 31)), "n"((P::P4 << 1) | (P::P3 >> 31)), "n"((P::P5 << 1) | (P::P4 >> 31)),
        "n"((P::P6 << 1) | (P::P5 >> 31)), "n"((P::P7 << 1) | (P::P6 >> 31)));
#pragma unroll
  for (int j = 0; j < 8; j++) r[j] = borrow ? s[j] : t[j];
}

// r = a - b, plus 2p if that borrowed.  Inputs < 2p.
template <class P>
__device__ __forceinline__ void sub_lazy(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  uint32_t d[8], borrow;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(borrow)
      : ZK_A_OPS(a), ZK_A_OPS(b));
  // conditional + 2p (mask form keeps it branch-free)
  const uint32_t mk = borrow;  // 0 or 0xffffffff
  asm("add.cc.u32  %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, %9;\n\t"
      "addc.cc.u32 %2, %2, %10;\n\t"
      "addc.cc.u32 %3, %3, %11;\n\t"
      "addc.cc.u32 %4, %4, %12;\n\t"
      "addc.cc.u32 %5, %5, %13;\n\t"
      "addc.cc.u32 %6, %6, %14;\n\t"
      "addc.u32    %7, %7, %15;"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]), "+r"(d[7])
      : "r"(mk & (uint32_t)(P::P0 << 1)), "r"(mk & ((P::P1 << 1) | (P::P0 >> 31))), "r"(mk & ((P::P2 << 1) | (P::P1 >> 31))),
        "r"(mk & ((P::P3 << 1) | (P::P2 >> 31))), "r"(mk & ((P::P4 << 1) | (P::P3 >> 31))),
        "r"(mk & ((P::P5 << 1) | (P::P4 >> 31))), "r"(mk & ((P::P6 << 1) | (P::P5 >> 31))),
        "r"(mk & ((P::P7 << 1) | (P::P6 >> 31))));
#pragma unroll
  for (int j = 0; j < 8; j++) r[j] = d[j];
}

// Reduce a value < 2p to canonical [0, p).
template <class P>
__device__ __forceinline__ void reduce_once(uint32_t r[8], const uint32_t a[8]) {
  uint32_t t[8], borrow;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7]), "=r"(borrow)
      : ZK_A_OPS(a), "n"(P::P0), "n"(P::P1), "n"(P::P2), "n"(P::P3), "n"(P::P4), "n"(P::P5), "n"(P::P6), "n"(P::P7));
#pragma unroll
  for (int j = 0; j < 8; j++) r[j] = borrow ? a[j] : t[j];
}

// ---- canonical forms (inputs < p, outputs < p) ---------------------------
template <class P>
__device__ __forceinline__ void mul(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  uint32_t t[8];
  mul_lazy<P>(t, a, b);
  reduce_once<P>(r, t);
}
template <class P>
__device__ __forceinline__ void sqr(uint32_t r[8], const uint32_t a[8]) {
  mul<P>(r, a, a);
}
template <class P>
__device__ __forceinline__ void add(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  uint32_t s[8];
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7])
      : ZK_A_OPS(a), ZK_A_OPS(b));
  reduce_once<P>(r, s);
}
template <class P>
__device__ __forceinline__ void sub(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  uint32_t d[8], borrow;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(borrow)
      : ZK_A_OPS(a), ZK_A_OPS(b));
  const uint32_t mk = borrow;
  asm("add.cc.u32  %0, %0, %8;\n\t"
      "addc.cc.u32 %1, %1, %9;\n\t"
      "addc.cc.u32 %2, %2, %10;\n\t"
      "addc.cc.u32 %3, %3, %11;\n\t"
      "addc.cc.u32 %4, %4, %12;\n\t"
      "addc.cc.u32 %5, %5, %13;\n\t"
      "addc.cc.u32 %6, %6, %14;\n\t"
      "addc.u32    %7, %7, %15;"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]), "+r"(d[7])
      : "r"(mk & P::P0), "r"(mk & P::P1), "r"(mk & P::P2), "r"(mk & P::P3), "r"(mk & P::P4), "r"(mk & P::P5),
        "r"(mk & P::P6), "r"(mk & P::P7));
#pragma unroll
  for (int j = 0; j < 8; j++) r[j] = d[j];
}
template <class P>
__device__ __forceinline__ void dbl(uint32_t r[8], const uint32_t a[8]) {
  add<P>(r, a, a);
}

__device__ __forceinline__ bool is_zero(const uint32_t a[8]) {
  return (a[0] | a[1] | a[2] | a[3] | a[4] | a[5] | a[6] | a[7]) == 0;
}
__device__ __forceinline__ bool eq(const uint32_t a[8], const uint32_t b[8]) {
  return ((a[0] ^ b[0]) | (a[1] ^ b[1]) | (a[2] ^ b[2]) | (a[3] ^ b[3]) | (a[4] ^ b[4]) | (a[5] ^ b[5]) |
          (a[6] ^ b[6]) | (a[7] ^ b[7])) == 0;
}
template <class P>
__device__ __forceinline__ void set_one(uint32_t r[8]) {
  r[0] = P::O0; r[1] = P::O1; r[2] = P::O2; r[3] = P::O3;
  r[4] = P::O4; r[5] = P::O5; r[6] = P::O6; r[7] = P::O7;
}
__device__ __forceinline__ void set_zero(uint32_t r[8]) {
#pragma unroll
  for (int j = 0; j < 8; j++) r[j] = 0;
}
__device__ __forceinline__ void cpy(uint32_t r[8], const uint32_t a[8]) {
#pragma unroll
  for (int j = 0; j < 8; j++) r[j] = a[j];
}

// a^e for a small exponent (canonical inputs), square-and-multiply
template <class P>
__device__ __forceinline__ void pow_u64(uint32_t r[8], const uint32_t a[8], uint64_t e) {
  uint32_t acc[8], base[8];
  set_one<P>(acc);
  cpy(base, a);
  while (e) {
    if (e & 1) mul<P>(acc, acc, base);
    e >>= 1;
    if (e) sqr<P>(base, base);
  }
  cpy(r, acc);
}

// ---- reduced-radix Montgomery product (9 limbs of 29 bits, R' = 2^261) ----
// Products of 29-bit limbs are < 2^58, so a 64-bit column accumulator takes
// every partial product of a column (at most 18, < 2^62.2) through one
// mad.wide.u32 each, with no carry chain; carries are resolved once per
// row (T[i+1] += T[i] >> 29).  It computes a*b*2^-261 mod p, so one operand
// is kept in "R' form" (x * 2^261 mod p): R-form data (x * 2^256) times an
// R'-form constant gives R-form data.  Inputs < 2p give a result < 2p
// (4p^2 / 2^261 < p / 32).
constexpr uint32_t M29 = (1u << 29) - 1;

__device__ __forceinline__ void split29(uint32_t l[9], const uint32_t a[8]) {
  l[0] = a[0] & M29;
  l[1] = __funnelshift_r(a[0], a[1], 29) & M29;
  l[2] = __funnelshift_r(a[1], a[2], 26) & M29;
  l[3] = __funnelshift_r(a[2], a[3], 23) & M29;
  l[4] = __funnelshift_r(a[3], a[4], 20) & M29;
  l[5] = __funnelshift_r(a[4], a[5], 17) & M29;
  l[6] = __funnelshift_r(a[5], a[6], 14) & M29;
  l[7] = __funnelshift_r(a[6], a[7], 11) & M29;
  l[8] = a[7] >> 8;
}

__device__ __forceinline__ void pack29(uint32_t w[8], const uint32_t l[9]) {
  w[0] = l[0] | (l[1] << 29);
  w[1] = (l[1] >> 3) | (l[2] << 26);
  w[2] = (l[2] >> 6) | (l[3] << 23);
  w[3] = (l[3] >> 9) | (l[4] << 20);
  w[4] = (l[4] >> 12) | (l[5] << 17);
  w[5] = (l[5] >> 15) | (l[6] << 14);
  w[6] = (l[6] >> 18) | (l[7] << 11);
  w[7] = (l[7] >> 21) | (l[8] << 8);
}

// 29-bit limb j of the modulus, and -p^-1 mod 2^29
template <class P>
__host__ __device__ constexpr uint32_t p29(int j) {
  return j == 0   ? (P::P0 & M29)
         : j == 1 ? (((P::P0 >> 29) | (P::P1 << 3)) & M29)
         : j == 2 ? (((P::P1 >> 26) | (P::P2 << 6)) & M29)
         : j == 3 ? (((P::P2 >> 23) | (P::P3 << 9)) & M29)
         : j == 4 ? (((P::P3 >> 20) | (P::P4 << 12)) & M29)
         : j == 5 ? (((P::P4 >> 17) | (P::P5 << 15)) & M29)
         : j == 6 ? (((P::P5 >> 14) | (P::P6 << 18)) & M29)
         : j == 7 ? (((P::P6 >> 11) | (P::P7 << 21)) & M29)
                  : (P::P7 >> 8);
}
template <class P>
__host__ __device__ constexpr uint32_t inv29() {
  return P::INV & M29;  // -p^-1 mod 2^32 reduced mod 2^29
}

// r = a * b' * 2^-261 mod p, limbs given pre-split (al, bl < 2^29 each,
// values < 2p); result as 9 normalised limbs.
template <class P>
__device__ __forceinline__ void mul29_limbs(uint32_t rl[9], const uint32_t al[9], const uint32_t bl[9]) {
  uint64_t T[17];
#pragma unroll
  for (int k = 0; k < 17; k++) T[k] = 0;
#pragma unroll
  for (int i = 0; i < 9; i++) {
#pragma unroll
    for (int j = 0; j < 9; j++) T[i + j] += (uint64_t)al[j] * bl[i];
    const uint32_t m = ((uint32_t)T[i] * inv29<P>()) & M29;
#pragma unroll
    for (int j = 0; j < 9; j++) T[i + j] += (uint64_t)m * p29<P>(j);
    T[i + 1] += T[i] >> 29;
  }
  uint64_t c = 0;
#pragma unroll
  for (int k = 9; k < 17; k++) {
    const uint64_t v = T[k] + c;
    rl[k - 9] = (uint32_t)v & M29;
    c = v >> 29;
  }
  rl[8] = (uint32_t)c;
}

// Same product in column (product-scanning) order: column k collects
// a_j b_(k-j) and m_j p_(k-j) in one 64-bit accumulator (< 18 * 2^58 + 2^35),
// so only that accumulator and the 9 quotient digits m_j stay live
// (register-light; measured a little faster than the row order).
template <class P>
__device__ __forceinline__ void mul29_cols(uint32_t rl[9], const uint32_t al[9], const uint32_t bl[9]) {
  uint32_t m[9];
  uint64_t acc = 0;
#pragma unroll
  for (int k = 0; k < 17; k++) {
#pragma unroll
    for (int j = 0; j < 9; j++) {
      const int i = k - j;
      if (i >= 0 && i < 9) acc += (uint64_t)al[j] * bl[i];
    }
#pragma unroll
    for (int j = 0; j < 9; j++) {
      const int i = k - j;
      if (j < k && i >= 0 && i < 9) acc += (uint64_t)m[j] * p29<P>(i);
    }
    if (k < 9) {
      m[k] = ((uint32_t)acc * inv29<P>()) & M29;
      acc += (uint64_t)m[k] * p29<P>(0);
      acc >>= 29;  // low 29 bits are zero
    } else {
      rl[k - 9] = (uint32_t)acc & M29;
      acc >>= 29;
    }
  }
  rl[8] = (uint32_t)acc;
}

// a (8 words, R form) times a pre-split R'-form constant b (9 limbs)
template <class P>
__device__ __forceinline__ void mul_r29_pre(uint32_t r[8], const uint32_t a[8], const uint32_t bl[9]) {
  uint32_t al[9], rl[9];
  split29(al, a);
  mul29_cols<P>(rl, al, bl);
  pack29(r, rl);
}

// 8-word interface: r = a * b' * 2^-261 (b' in R' form), lazy (< 2p).
template <class P>
__device__ __forceinline__ void mul_r29(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  uint32_t al[9], bl[9], rl[9];
  split29(al, a);
  split29(bl, b);
  mul29_cols<P>(rl, al, bl);
  pack29(r, rl);
}

template <class P>
__device__ __forceinline__ void set_one_r29(uint32_t r[8]) {
  r[0] = P::Q0; r[1] = P::Q1; r[2] = P::Q2; r[3] = P::Q3;
  r[4] = P::Q4; r[5] = P::Q5; r[6] = P::Q6; r[7] = P::Q7;
}
// a^e with a and the result in R' form (canonical)
template <class P>
__device__ __forceinline__ void pow_u64_r29(uint32_t r[8], const uint32_t a[8], uint64_t e) {
  uint32_t acc[8], base[8];
  set_one_r29<P>(acc);
  cpy(base, a);
  while (e) {
    if (e & 1) mul_r29<P>(acc, acc, base);
    e >>= 1;
    if (e) mul_r29<P>(base, base, base);
  }
  reduce_once<P>(r, acc);
}

// ---- FP64 product: 5 limbs of 52 bits in doubles, R' = 2^260 --------------
// The hot-path product.  Limbs are exact integers < 2^52 held in doubles;
// each 52 x 52-bit partial product is split exactly into its high and low
// 52-bit halves by two fused multiply-adds rounded toward zero:
//   h = fma_rz(a, b, 2^104)             = 2^104 + floor(ab / 2^52) 2^52
//   l = fma_rz(a, b, 2^104 + 2^52 - h)  = 2^52  + (ab mod 2^52)
// Every value involved is exactly representable (the subtraction
// 2^104 + 2^52 - h too), so nothing is rounded.  The IEEE bit patterns of h
// and l are integers with a constant bias: bits(h) - bits(2^104) =
// floor(ab / 2^52) and bits(l) - bits(2^52) = ab mod 2^52.  They are summed
// per column (product scanning) in 64-bit integers, the biases removed once
// per column, and the Montgomery quotient digit m_k = t_k (-p^-1) mod 2^52
// comes from an integer multiply; its products m_k p_j are split the same
// way.  The result is a b 2^-260 mod p, lazily reduced: inputs < 2p give an
// output < 2p (4p^2 / 2^260 < p).  This moves the 256-bit product from the
// 32-bit IMAD pipe (mul29_cols: 81 + 81 word products as lo/hi pairs) to
// the FP64 pipe (50 + 50 DFMA, 50 exact DADD) with the column sums on the
// integer ALU; measured 1.4x the product rate of mul29_cols on B200.  The
// method is the one published by Emmart, Zheng and Weems, "Faster Modular
// Exponentiation Using Double Precision Floating Point Arithmetic on the
// GPU" (ARITH 2018).
constexpr uint64_t M52 = (1ull << 52) - 1;
constexpr double D2P52 = 4503599627370496.0;                      // 2^52
constexpr double D2P104 = 20282409603651670423947251286016.0;     // 2^104
constexpr double D2P104_52 = 20282409603651674927546878656512.0;  // 2^104 + 2^52
constexpr uint64_t BITS_2P52 = 0x4330000000000000ull;
constexpr uint64_t BITS_2P104 = 0x4670000000000000ull;

template <class P>
__host__ __device__ constexpr uint64_t pword64(int k) {
  return k == 0   ? ((uint64_t)P::P1 << 32 | P::P0)
         : k == 1 ? ((uint64_t)P::P3 << 32 | P::P2)
         : k == 2 ? ((uint64_t)P::P5 << 32 | P::P4)
                  : ((uint64_t)P::P7 << 32 | P::P6);
}
// limb j (52 bits) of the modulus, as a double
template <class P>
__host__ __device__ constexpr double p52(int j) {
  return (double)(j == 0   ? (pword64<P>(0) & M52)
                  : j == 1 ? ((pword64<P>(0) >> 52 | pword64<P>(1) << 12) & M52)
                  : j == 2 ? ((pword64<P>(1) >> 40 | pword64<P>(2) << 24) & M52)
                  : j == 3 ? ((pword64<P>(2) >> 28 | pword64<P>(3) << 36) & M52)
                           : (pword64<P>(3) >> 16));
}
// -p^-1 mod 2^52 (Newton iteration on the low word)
template <class P>
__host__ __device__ constexpr uint64_t pinv52() {
  uint64_t x = 1;
  for (int i = 0; i < 7; i++) x *= 2 - pword64<P>(0) * x;
  return (0 - x) & M52;
}

__device__ __forceinline__ double dbl_of_limb(uint64_t v) {  // v < 2^52 -> (double)v, exactly
  return __longlong_as_double((long long)(v | BITS_2P52)) - D2P52;
}
__device__ __forceinline__ uint64_t bits_of(double x) { return (uint64_t)__double_as_longlong(x); }

__device__ __forceinline__ void split52(double l[5], const uint32_t a[8]) {
  const uint64_t x0 = (uint64_t)a[1] << 32 | a[0], x1 = (uint64_t)a[3] << 32 | a[2];
  const uint64_t x2 = (uint64_t)a[5] << 32 | a[4], x3 = (uint64_t)a[7] << 32 | a[6];
  l[0] = dbl_of_limb(x0 & M52);
  l[1] = dbl_of_limb((x0 >> 52 | x1 << 12) & M52);
  l[2] = dbl_of_limb((x1 >> 40 | x2 << 24) & M52);
  l[3] = dbl_of_limb((x2 >> 28 | x3 << 36) & M52);
  l[4] = dbl_of_limb(x3 >> 16);
}
__device__ __forceinline__ void pack52(uint32_t r[8], const uint64_t l[5]) {
  const uint64_t x0 = l[0] | l[1] << 52, x1 = l[1] >> 12 | l[2] << 40;
  const uint64_t x2 = l[2] >> 24 | l[3] << 28, x3 = l[3] >> 36 | l[4] << 16;
  r[0] = (uint32_t)x0; r[1] = (uint32_t)(x0 >> 32); r[2] = (uint32_t)x1; r[3] = (uint32_t)(x1 >> 32);
  r[4] = (uint32_t)x2; r[5] = (uint32_t)(x2 >> 32); r[6] = (uint32_t)x3; r[7] = (uint32_t)(x3 >> 32);
}

// index pairs (j, i), 0 <= i, j < 5, with i + j = k
__host__ __device__ constexpr int npairs5(int k) { return k < 0 || k > 8 ? 0 : (k <= 4 ? k + 1 : 9 - k); }
// quotient terms m_j p_i with j + i = k (m_k p_0 included for k < 5)
__host__ __device__ constexpr int nquot5(int k) { return k < 0 ? 0 : (k < 5 ? k + 1 : npairs5(k)); }

// a * b * 2^-260 mod p as 5 normalised 52-bit limbs (a, b < 2p as limbs)
template <class P>
__device__ __forceinline__ void mul52_cols(uint64_t rl[5], const double a[5], const double b[5]) {
  double m[5];
  uint64_t cur = 0, nxt = 0;
#pragma unroll
  for (int k = 0; k < 10; k++) {
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const int i = k - j;
      if (i >= 0 && i < 5) {
        const double h = __fma_rz(a[j], b[i], D2P104);
        const double l = __fma_rz(a[j], b[i], D2P104_52 - h);
        cur += bits_of(l);
        nxt += bits_of(h);
      }
    }
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const int i = k - j;
      if (j < k && i >= 0 && i < 5) {
        const double h = __fma_rz(m[j], p52<P>(i), D2P104);
        const double l = __fma_rz(m[j], p52<P>(i), D2P104_52 - h);
        cur += bits_of(l);
        nxt += bits_of(h);
      }
    }
    // biases: this column's low halves so far, and the high halves the
    // previous column passed on (they arrived in `cur` with the carry)
    const uint64_t nlo = (uint64_t)(npairs5(k) + (k < 5 ? k : npairs5(k)));
    const uint64_t nhi = (uint64_t)(npairs5(k - 1) + nquot5(k - 1));
    cur -= nlo * BITS_2P52 + nhi * BITS_2P104;
    if (k < 5) {
      m[k] = dbl_of_limb(((cur & M52) * pinv52<P>()) & M52);
      const double h = __fma_rz(m[k], p52<P>(0), D2P104);
      const double l = __fma_rz(m[k], p52<P>(0), D2P104_52 - h);
      cur += bits_of(l) - BITS_2P52;  // now a multiple of 2^52
      nxt += bits_of(h);
    } else {
      rl[k - 5] = cur & M52;
    }
    cur = nxt + (cur >> 52);
    nxt = 0;
  }
}

// 8-word interface: r = a * b' * 2^-260 (b' in R' form), lazy (< 2p)
template <class P>
__device__ __forceinline__ void mul_rp(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  double al[5], bl[5];
  uint64_t rl[5];
  split52(al, a);
  split52(bl, b);
  mul52_cols<P>(rl, al, bl);
  pack52(r, rl);
}
// a (8 words) times a pre-split R'-form constant
template <class P>
__device__ __forceinline__ void mul_rp_pre(uint32_t r[8], const uint32_t a[8], const double bl[5]) {
  double al[5];
  uint64_t rl[5];
  split52(al, a);
  mul52_cols<P>(rl, al, bl);
  pack52(r, rl);
}
// The same product as a call of one out-of-line function: operands and
// result pass by value (in registers), so a kernel that runs many products
// keeps one copy of the product's ~360 instructions in the instruction cache
// instead of one inlined copy per call site.
struct Fe8 {
  uint32_t w[8];
};
template <class P>
__device__ __noinline__ Fe8 mul_rp_call(const Fe8 a, const Fe8 b) {
  Fe8 r;
  mul_rp<P>(r.w, a.w, b.w);
  return r;
}
template <class P>
__device__ __forceinline__ void mul_rp_out(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
  Fe8 av, bv;
#pragma unroll
  for (int k = 0; k < 8; k++) av.w[k] = a[k], bv.w[k] = b[k];
  const Fe8 rv = mul_rp_call<P>(av, bv);
#pragma unroll
  for (int k = 0; k < 8; k++) r[k] = rv.w[k];
}
template <class P>
__device__ __forceinline__ void set_one_rp(uint32_t r[8]) {
  r[0] = P::D0; r[1] = P::D1; r[2] = P::D2; r[3] = P::D3;
  r[4] = P::D4; r[5] = P::D5; r[6] = P::D6; r[7] = P::D7;
}
// a^e with a and the result in R' form (canonical)
template <class P>
__device__ __forceinline__ void pow_u64_rp(uint32_t r[8], const uint32_t a[8], uint64_t e) {
  uint32_t acc[8], base[8];
  set_one_rp<P>(acc);
  cpy(base, a);
  while (e) {
    if (e & 1) mul_rp<P>(acc, acc, base);
    e >>= 1;
    if (e) mul_rp<P>(base, base, base);
  }
  reduce_once<P>(r, acc);
}

// ---- global memory element access (32 B = one sector, two 16 B vectors) --
__device__ __forceinline__ void ld_fe(uint32_t r[8], const fe* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4 x = q[0], y = q[1];
  r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
  r[4] = y.x; r[5] = y.y; r[6] = y.z; r[7] = y.w;
}
__device__ __forceinline__ void ld_fe_nc(uint32_t r[8], const fe* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4 x = __ldg(q), y = __ldg(q + 1);
  r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
  r[4] = y.x; r[5] = y.y; r[6] = y.z; r[7] = y.w;
}
// through L2 only: data another CTA of the same launch may have written
__device__ __forceinline__ void ld_fe_cg(uint32_t r[8], const fe* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4 x = __ldcg(q), y = __ldcg(q + 1);
  r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
  r[4] = y.x; r[5] = y.y; r[6] = y.z; r[7] = y.w;
}
__device__ __forceinline__ void st_fe(fe* p, const uint32_t r[8]) {
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4(r[0], r[1], r[2], r[3]);
  q[1] = make_uint4(r[4], r[5], r[6], r[7]);
}

}  // namespace zk
