/*
 * zkoracle.h — CPU oracle for the halo2/BN256 NTT + MSM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests, the smoke
 * entry and the benchmark's CPU-baseline leg may call it; the product path
 * (libzkgpu.so) never links or calls it.
 *
 * It restates, in plain C, the CPU algorithms the reference's callers use:
 *   - halo2 `best_fft` (bit-reverse + radix-2 DIT with the recursive split,
 *     twiddles w^i, i < n/2), `ifft` (best_fft with w^-1, then * divisor),
 *     `distribute_powers` (a[i] *= c^i) and the coeff -> extended coset LDE;
 *     the reference GPU path that replaces them is cuda/fft.cu:11-42 (serial
 *     DIT), :61-113 (four-step), :149-156 (ifft scaling), :223-232 (coset).
 *   - halo2 `best_multiexp` (per-thread chunk of windowed Pippenger with
 *     c = ceil(ln n) and 256/c+1 windows, then a sum of the chunk results);
 *     reference GPU restatement cuda/fft.cu:158-221, curve.cuh:108-297.
 *   - halo2 `generate_twiddle_lookup_table(omega, k, 10, true)`, the twiddle
 *     table the reference FFI takes (cuda/fft.cu:72-79, src/main.rs:128-138).
 * Field constants follow cuda/bn256.h:37-56.  Elements are 4 x u64
 * little-endian limbs in Montgomery form (R = 2^256), bit-identical to
 * halo2curves' Fr / Fq repr and to the reference's BigNum.
 *
 * halo2 itself (an unpinned external fork of halo2_proofs / halo2curves) is
 * not present and cannot be built here, so this is a restatement of its
 * published algorithm; it is pinned by known-answer tests and by fixtures
 * produced by the reference's own CUDA path (tests/golden/).
 */
#ifndef ZKORACLE_H
#define ZKORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- field: id 0 = Fr (scalar field r), 1 = Fq (base field q) ---------- */
void zko_field_mul(int fid, uint64_t out[4], const uint64_t a[4], const uint64_t b[4]);
void zko_field_add(int fid, uint64_t out[4], const uint64_t a[4], const uint64_t b[4]);
void zko_field_sub(int fid, uint64_t out[4], const uint64_t a[4], const uint64_t b[4]);
void zko_field_pow(int fid, uint64_t out[4], const uint64_t a[4], const uint64_t e[4]);
void zko_field_inv(int fid, uint64_t out[4], const uint64_t a[4]);
void zko_to_mont(int fid, uint64_t out[4], const uint64_t canonical[4]);
void zko_from_mont(int fid, uint64_t out[4], const uint64_t mont[4]);
/* vectorised: out[i] = a[i] * b[i] (Montgomery) */
void zko_field_mul_vec(int fid, uint64_t *out, const uint64_t *a, const uint64_t *b, size_t n, int threads);
/* out = sum_i a[i] * b[i] (Montgomery products, summed mod p) */
void zko_field_dot(int fid, uint64_t out[4], const uint64_t *a, const uint64_t *b, size_t n, int threads);
/* element-wise vector ops (extended-domain evaluations): out = a + b, a - b,
 * a * c (+ b if b != NULL) */
void zko_field_add_vec(int fid, uint64_t *out, const uint64_t *a, const uint64_t *b, size_t n, int threads);
void zko_field_sub_vec(int fid, uint64_t *out, const uint64_t *a, const uint64_t *b, size_t n, int threads);
void zko_field_axpy_vec(int fid, uint64_t *out, const uint64_t *a, const uint64_t c[4], const uint64_t *b, size_t n,
                        int threads);
/* halo2 divide_by_vanishing_poly on the coset g<w_ext>: ext[k] /= g^n w_ext^(n (k mod 2^(log_ext-log_n))) - 1 */
int zko_divide_by_vanishing(uint64_t *ext, uint32_t log_n, uint32_t log_ext, const uint64_t g[4],
                            const uint64_t omega_ext[4], int threads);

/* ---- seeded synthetic inputs ------------------------------------------- */
/* n uniform Fr elements in Montgomery form (each < r), counter-based so any
 * slice [start, start+n) of a stream is reproducible independently. */
void zko_rand_fr(uint64_t *out, size_t n, uint64_t seed, size_t start, int threads);
/* uniform small canonical values in [0, 2^bits) converted to Montgomery */
void zko_rand_fr_small(uint64_t *out, size_t n, uint64_t seed, size_t start, int bits, int threads);
/* n affine G1 points [k_i] * (1, 2) for seeded canonical k_i < r; k (if not
 * NULL) receives the k_i in Montgomery form so tests can use discrete logs. */
void zko_rand_bases(uint64_t *bases_xy, uint64_t *k_mont, size_t n, uint64_t seed, size_t start, int threads);

/* ---- NTT (halo2 semantics) -------------------------------------------- */
/* in place, natural order in and out: a[k] <- sum_i a[i] * omega^(i k) */
int zko_best_fft(uint64_t *a, const uint64_t omega[4], uint32_t log_n, int threads);
/* best_fft with omega_inv, then every element * divisor */
int zko_ifft(uint64_t *a, const uint64_t omega_inv[4], uint32_t log_n, const uint64_t divisor[4], int threads);
/* a[i] <- a[i] * c^i */
int zko_distribute_powers(uint64_t *a, size_t n, const uint64_t c[4], int threads);
/* halo2 coeff_to_extended with the g^i coset: ext[0..2^log_ext) <-
 * best_fft(zero-pad(a * g^i), omega_ext).  `a` (2^log_n) is not modified. */
int zko_coeff_to_extended(const uint64_t *a, uint32_t log_n, uint64_t *ext, uint32_t log_ext,
                          const uint64_t g[4], const uint64_t omega_ext[4], int threads);
/* halo2 generate_twiddle_lookup_table(omega, log_n, sparse_degree, with_last_level).
 * Returns the number of elements written (out may be NULL to query). */
size_t zko_twiddle_lut(uint64_t *out, const uint64_t omega[4], uint32_t log_n,
                       uint32_t sparse_degree, int with_last_level);
/* the 2^log_n-th root used by halo2: ROOT_OF_UNITY^(2^(28-log_n)), Montgomery */
int zko_omega(uint64_t out[4], uint32_t log_n);
/* O(n^2) DFT, for cross-checking best_fft at small n */
int zko_naive_dft(uint64_t *out, const uint64_t *a, size_t n, const uint64_t omega[4]);

/* ---- G1 (y^2 = x^3 + 3 over Fq) ---------------------------------------- */
/* affine points are (x, y) Montgomery, identity encoded as (0, 0);
 * jacobian points are (X, Y, Z), identity Z = 0. */
void zko_g1_normalize(uint64_t out_xy[8], const uint64_t jac[12]);
void zko_g1_scalar_mul(uint64_t out_xy[8], const uint64_t base_xy[8], const uint64_t scalar_mont[4]);
void zko_g1_add_affine(uint64_t out_xy[8], const uint64_t a_xy[8], const uint64_t b_xy[8]);
int  zko_g1_on_curve(const uint64_t xy[8]);
/* halo2 best_multiexp: sum_i scalars[i] * bases[i]; result normalised affine */
int zko_multiexp(uint64_t out_xy[8], const uint64_t *scalars_mont, const uint64_t *bases_xy,
                 size_t n, int threads);
/* double-and-add sum, for small-n cross-checks */
int zko_naive_msm(uint64_t out_xy[8], const uint64_t *scalars_mont, const uint64_t *bases_xy, size_t n);

#ifdef __cplusplus
}
#endif
#endif
