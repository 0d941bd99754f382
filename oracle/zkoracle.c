/*
 * zkoracle.c — CPU oracle (TEST INFRASTRUCTURE ONLY; see zkoracle.h).
 *
 * Plain C + OpenMP restatement of halo2's CPU path for the Fr NTT and the
 * G1 multiexp.  Nothing here is called by the product library.
 */
#include "zkoracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------ */
/* Field constants (cuda/bn256.h:37-56; re-derived and checked in tests)     */
/* ------------------------------------------------------------------------ */
typedef struct {
    u64 p[4];
    u64 inv;   /* -p^-1 mod 2^64 */
    u64 one[4];  /* R mod p */
    u64 r2[4];   /* R^2 mod p */
} field_t;

static const field_t FIELDS[2] = {
    { /* Fr, bn256.h:52-56 */
        {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
        0xc2e1f593efffffffULL,
        {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL},
        {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL},
    },
    { /* Fq, bn256.h:37-48 */
        {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
        0x87d20782e4866389ULL,
        {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL},
        {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL},
    },
};
#define FR (&FIELDS[0])
#define FQ (&FIELDS[1])

/* Fr::ROOT_OF_UNITY = 7^((r-1)/2^28), canonical (bn256.h:57, commented) */
static const u64 FR_ROOT_CANON[4] = {0xd34f1ed960c37c9cULL, 0x3215cf6dd39329c8ULL,
                                     0x98865ea93dd31f74ULL, 0x03ddb9f5166d18b7ULL};

static inline int geq4(const u64 a[4], const u64 b[4]) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] > b[i]) return 1;
        if (a[i] < b[i]) return 0;
    }
    return 1;
}
static inline int is_zero4(const u64 a[4]) { return (a[0] | a[1] | a[2] | a[3]) == 0; }
static inline int eq4(const u64 a[4], const u64 b[4]) {
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2] && a[3] == b[3];
}
static inline void cpy4(u64 d[4], const u64 s[4]) { d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; d[3] = s[3]; }

static inline u64 sub4(u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 borrow = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        r[i] = (u64)d;
        borrow = (u64)(d >> 64) & 1;
    }
    return borrow;
}
static inline u64 add4(u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 carry = 0;
    for (int i = 0; i < 4; i++) {
        u128 s = (u128)a[i] + b[i] + carry;
        r[i] = (u64)s;
        carry = (u64)(s >> 64);
    }
    return carry;
}

/* canonical modular add / sub (inputs < p) */
static inline void fadd(const field_t *F, u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 t[4];
    add4(t, a, b); /* p < 2^254: no carry out */
    if (geq4(t, F->p)) sub4(t, t, F->p);
    cpy4(r, t);
}
static inline void fsub(const field_t *F, u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 t[4];
    if (sub4(t, a, b)) add4(t, t, F->p);
    cpy4(r, t);
}
static inline void fdbl(const field_t *F, u64 r[4], const u64 a[4]) { fadd(F, r, a, a); }

/* CIOS Montgomery product a*b*R^-1 mod p, canonical output for inputs < p */
static inline void fmul(const field_t *F, u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u64 c = 0;
        for (int j = 0; j < 4; j++) {
            u128 s = (u128)a[j] * b[i] + t[j] + c;
            t[j] = (u64)s;
            c = (u64)(s >> 64);
        }
        u128 s = (u128)t[4] + c;
        t[4] = (u64)s;
        t[5] = (u64)(s >> 64);
        u64 m = t[0] * F->inv;
        s = (u128)m * F->p[0] + t[0];
        c = (u64)(s >> 64);
        for (int j = 1; j < 4; j++) {
            s = (u128)m * F->p[j] + t[j] + c;
            t[j - 1] = (u64)s;
            c = (u64)(s >> 64);
        }
        s = (u128)t[4] + c;
        t[3] = (u64)s;
        t[4] = t[5] + (u64)(s >> 64);
    }
    u64 res[4] = {t[0], t[1], t[2], t[3]};
    if (t[4] || geq4(res, F->p)) sub4(res, res, F->p);
    cpy4(r, res);
}
static inline void fsqr(const field_t *F, u64 r[4], const u64 a[4]) { fmul(F, r, a, a); }

/* a^e for a canonical exponent e (4 x u64, little endian) */
static void fpow(const field_t *F, u64 r[4], const u64 a[4], const u64 e[4]) {
    u64 acc[4];
    cpy4(acc, F->one);
    for (int i = 3; i >= 0; i--)
        for (int b = 63; b >= 0; b--) {
            fsqr(F, acc, acc);
            if ((e[i] >> b) & 1) fmul(F, acc, acc, a);
        }
    cpy4(r, acc);
}
static void fpow_u64(const field_t *F, u64 r[4], const u64 a[4], u64 e) {
    u64 ee[4] = {e, 0, 0, 0};
    fpow(F, r, a, ee);
}
static void finv(const field_t *F, u64 r[4], const u64 a[4]) {
    u64 e[4];
    cpy4(e, F->p);
    e[0] -= 2; /* p - 2, p odd and p[0] > 2 */
    fpow(F, r, a, e);
}

static const field_t *fld(int fid) { return fid ? FQ : FR; }

void zko_field_mul(int fid, u64 out[4], const u64 a[4], const u64 b[4]) { fmul(fld(fid), out, a, b); }
void zko_field_add(int fid, u64 out[4], const u64 a[4], const u64 b[4]) { fadd(fld(fid), out, a, b); }
void zko_field_sub(int fid, u64 out[4], const u64 a[4], const u64 b[4]) { fsub(fld(fid), out, a, b); }
void zko_field_pow(int fid, u64 out[4], const u64 a[4], const u64 e[4]) { fpow(fld(fid), out, a, e); }
void zko_field_inv(int fid, u64 out[4], const u64 a[4]) { finv(fld(fid), out, a); }
void zko_to_mont(int fid, u64 out[4], const u64 c[4]) { fmul(fld(fid), out, c, fld(fid)->r2); }
void zko_from_mont(int fid, u64 out[4], const u64 m[4]) {
    static const u64 one[4] = {1, 0, 0, 0};
    fmul(fld(fid), out, m, one);
}
void zko_field_mul_vec(int fid, u64 *out, const u64 *a, const u64 *b, size_t n, int threads) {
    const field_t *F = fld(fid);
#pragma omp parallel for num_threads(threads > 0 ? threads : omp_get_max_threads()) schedule(static)
    for (size_t i = 0; i < n; i++) fmul(F, out + 4 * i, a + 4 * i, b + 4 * i);
}

static int nthreads(int threads) { return threads > 0 ? threads : omp_get_max_threads(); }

/* Element-wise vector ops on extended-domain evaluations (halo2's quotient
 * step combines polynomials in ExtendedLagrangeCoeff form this way:
 * Polynomial Mul / Add / Sub and scalar Mul, halo2_proofs/src/poly.rs). */
void zko_field_add_vec(int fid, u64 *out, const u64 *a, const u64 *b, size_t n, int threads) {
    const field_t *F = fld(fid);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (size_t i = 0; i < n; i++) fadd(F, out + 4 * i, a + 4 * i, b + 4 * i);
}
void zko_field_sub_vec(int fid, u64 *out, const u64 *a, const u64 *b, size_t n, int threads) {
    const field_t *F = fld(fid);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (size_t i = 0; i < n; i++) fsub(F, out + 4 * i, a + 4 * i, b + 4 * i);
}
/* out = a * c (+ b when b is not NULL), c one element */
void zko_field_axpy_vec(int fid, u64 *out, const u64 *a, const u64 c[4], const u64 *b, size_t n, int threads) {
    const field_t *F = fld(fid);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (size_t i = 0; i < n; i++) {
        u64 t[4];
        fmul(F, t, a + 4 * i, c);
        if (b) fadd(F, t, t, b + 4 * i);
        cpy4(out + 4 * i, t);
    }
}

/* halo2 EvaluationDomain::divide_by_vanishing_poly (halo2_proofs/src/poly/
 * domain.rs, the external halo2 fork the reference's callers use): the
 * vanishing polynomial t(X) = X^n - 1 takes only 2^(log_ext - log_n) distinct
 * values on the coset g * <w_ext>, t_j = g^n * w_ext^(n j) - 1; they are
 * inverted once and ext[k] is multiplied by 1 / t_(k mod 2^(log_ext-log_n)).
 * Returns -1 (nothing changed) when some t_j is zero (g^n in <w_ext^n>). */
int zko_divide_by_vanishing(u64 *ext, uint32_t log_n, uint32_t log_ext, const u64 g[4], const u64 omega_ext[4],
                            int threads) {
    if (log_ext < log_n || log_ext - log_n > 16) return -1;
    const size_t n = (size_t)1 << log_n, N = (size_t)1 << log_ext, J = (size_t)1 << (log_ext - log_n);
    u64 *tinv = (u64 *)malloc(sizeof(u64) * 4 * J);
    u64 gn[4], step[4], cur[4];
    fpow_u64(FR, gn, g, n);
    fpow_u64(FR, step, omega_ext, n);
    cpy4(cur, gn);
    for (size_t j = 0; j < J; j++) {
        u64 t[4];
        fsub(FR, t, cur, FR->one);
        if (is_zero4(t)) {
            free(tinv);
            return -1;
        }
        finv(FR, tinv + 4 * j, t);
        fmul(FR, cur, cur, step);
    }
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (size_t k = 0; k < N; k++) fmul(FR, ext + 4 * k, ext + 4 * k, tinv + 4 * (k & (J - 1)));
    free(tinv);
    return 0;
}

void zko_field_dot(int fid, u64 out[4], const u64 *a, const u64 *b, size_t n, int threads) {
    const field_t *F = fld(fid);
    int T = nthreads(threads);
    u64 *part = (u64 *)calloc((size_t)T * 4, sizeof(u64));
#pragma omp parallel num_threads(T)
    {
        u64 acc[4] = {0, 0, 0, 0}, t[4];
        int id = omp_get_thread_num();
#pragma omp for schedule(static)
        for (size_t i = 0; i < n; i++) {
            fmul(F, t, a + 4 * i, b + 4 * i);
            fadd(F, acc, acc, t);
        }
        cpy4(part + 4 * id, acc);
    }
    u64 acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < T; i++) fadd(F, acc, acc, part + 4 * i);
    cpy4(out, acc);
    free(part);
}

/* ------------------------------------------------------------------------ */
/* Seeded synthetic inputs                                                   */
/* ------------------------------------------------------------------------ */
static inline u64 mix64(u64 z) { /* SplitMix64 finaliser */
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static inline u64 rnd(u64 seed, u64 idx, u64 attempt, u64 word) {
    u64 z = seed * 0x9e3779b97f4a7c15ULL + 0x632be59bd9b4e019ULL;
    z = mix64(z ^ (idx * 0xd1b54a32d192ed03ULL));
    z = mix64(z ^ (attempt * 0x8cb92ba72f3d8dd7ULL + word * 0xaf251af3b0f025b5ULL));
    return z;
}
/* uniform in [0, r) by rejection on 254-bit draws */
static void rand_below_r(u64 out[4], u64 seed, u64 idx) {
    for (u64 att = 0;; att++) {
        u64 v[4];
        for (int w = 0; w < 4; w++) v[w] = rnd(seed, idx, att, w);
        v[3] &= (1ULL << 62) - 1;
        if (!geq4(v, FR->p)) {
            cpy4(out, v);
            return;
        }
    }
}

void zko_rand_fr(u64 *out, size_t n, u64 seed, size_t start, int threads) {
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (size_t i = 0; i < n; i++) rand_below_r(out + 4 * i, seed, start + i);
}

void zko_rand_fr_small(u64 *out, size_t n, u64 seed, size_t start, int bits, int threads) {
    u64 mask = bits >= 64 ? ~0ULL : ((1ULL << bits) - 1);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (size_t i = 0; i < n; i++) {
        u64 c[4] = {rnd(seed ^ 0x5eed5ca1a7ULL, start + i, 0, 0) & mask, 0, 0, 0};
        fmul(FR, out + 4 * i, c, FR->r2);
    }
}

/* ------------------------------------------------------------------------ */
/* NTT: halo2 best_fft                                                       */
/* ------------------------------------------------------------------------ */
static inline size_t bitrev(size_t x, unsigned bits) {
    size_t r = 0;
    for (unsigned i = 0; i < bits; i++) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

/* butterfly: (a, b) <- (a + t, a - t), t = b * w  (w == NULL: twiddle one) */
static inline void bfly(u64 *a, u64 *b, const u64 *w) {
    u64 t[4];
    if (w)
        fmul(FR, t, b, w);
    else
        cpy4(t, b);
    fsub(FR, b, a, t);
    fadd(FR, a, a, t);
}

/* halo2 recursive_butterfly_arithmetic(a, n, twiddle_chunk, twiddles):
 * both halves first (in parallel), then the combining butterflies with
 * twiddles[i * twiddle_chunk].  `par` is the remaining task-spawn depth. */
static void rec_butterfly(u64 *a, size_t n, size_t twiddle_chunk, const u64 *tw, int par) {
    if (n == 2) {
        bfly(a, a + 4, NULL);
        return;
    }
    size_t h = n / 2;
    if (par > 0) {
#pragma omp task untied
        rec_butterfly(a, h, twiddle_chunk * 2, tw, par - 1);
#pragma omp task untied
        rec_butterfly(a + 4 * h, h, twiddle_chunk * 2, tw, par - 1);
#pragma omp taskwait
        /* combine in parallel chunks (same butterflies as the serial loop) */
        const size_t CH = 4096;
        for (size_t s = 0; s < h; s += CH) {
#pragma omp task firstprivate(s)
            {
                size_t e = s + CH < h ? s + CH : h;
                for (size_t i = s; i < e; i++) bfly(a + 4 * i, a + 4 * (i + h), i ? tw + 4 * (i * twiddle_chunk) : NULL);
            }
        }
#pragma omp taskwait
    } else {
        rec_butterfly(a, h, twiddle_chunk * 2, tw, 0);
        rec_butterfly(a + 4 * h, h, twiddle_chunk * 2, tw, 0);
        bfly(a, a + 4 * h, NULL);
        for (size_t i = 1; i < h; i++) bfly(a + 4 * i, a + 4 * (i + h), tw + 4 * (i * twiddle_chunk));
    }
}

int zko_best_fft(u64 *a, const u64 omega[4], uint32_t log_n, int threads) {
    if (log_n > 30) return -1;
    size_t n = (size_t)1 << log_n;
    int T = nthreads(threads);
    if (n == 1) return 0;
    /* bit-reverse permutation */
#pragma omp parallel for num_threads(T) schedule(static)
    for (size_t k = 0; k < n; k++) {
        size_t rk = bitrev(k, log_n);
        if (k < rk) {
            u64 t[4];
            cpy4(t, a + 4 * k);
            cpy4(a + 4 * k, a + 4 * rk);
            cpy4(a + 4 * rk, t);
        }
    }
    /* twiddles w^i, i < n/2 (parallel scan in chunks, as halo2's parallelize) */
    size_t h = n / 2;
    u64 *tw = (u64 *)malloc(sizeof(u64) * 4 * (h ? h : 1));
    if (!tw) return -2;
    const size_t CH = 1 << 14;
#pragma omp parallel for num_threads(T) schedule(static)
    for (size_t s = 0; s < h; s += CH) {
        u64 w[4];
        fpow_u64(FR, w, omega, s);
        size_t e = s + CH < h ? s + CH : h;
        for (size_t i = s; i < e; i++) {
            cpy4(tw + 4 * i, w);
            fmul(FR, w, w, omega);
        }
    }
    int par = 0;
    while ((1 << par) < 4 * T && par < 20) par++;
#pragma omp parallel num_threads(T)
#pragma omp single
    rec_butterfly(a, n, 1, tw, par);
    free(tw);
    return 0;
}

int zko_ifft(u64 *a, const u64 omega_inv[4], uint32_t log_n, const u64 divisor[4], int threads) {
    int rc = zko_best_fft(a, omega_inv, log_n, threads);
    if (rc) return rc;
    size_t n = (size_t)1 << log_n;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (size_t i = 0; i < n; i++) fmul(FR, a + 4 * i, a + 4 * i, divisor);
    return 0;
}

int zko_distribute_powers(u64 *a, size_t n, const u64 c[4], int threads) {
    const size_t CH = 1 << 14;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (size_t s = 0; s < n; s += CH) {
        u64 w[4];
        fpow_u64(FR, w, c, s);
        size_t e = s + CH < n ? s + CH : n;
        for (size_t i = s; i < e; i++) {
            fmul(FR, a + 4 * i, a + 4 * i, w);
            fmul(FR, w, w, c);
        }
    }
    return 0;
}

int zko_coeff_to_extended(const u64 *a, uint32_t log_n, u64 *ext, uint32_t log_ext, const u64 g[4],
                          const u64 omega_ext[4], int threads) {
    if (log_ext < log_n) return -1;
    size_t n = (size_t)1 << log_n, N = (size_t)1 << log_ext;
    memcpy(ext, a, sizeof(u64) * 4 * n);
    memset(ext + 4 * n, 0, sizeof(u64) * 4 * (N - n));
    zko_distribute_powers(ext, n, g, threads);
    return zko_best_fft(ext, omega_ext, log_ext, threads);
}

size_t zko_twiddle_lut(u64 *out, const u64 omega[4], uint32_t log_n, uint32_t sparse_degree, int with_last_level) {
    if (sparse_degree >= log_n) { /* dense table: w^i, i < n */
        size_t n = (size_t)1 << log_n;
        if (out) {
            u64 w[4];
            cpy4(w, FR->one);
            for (size_t i = 0; i < n; i++) {
                cpy4(out + 4 * i, w);
                fmul(FR, w, w, omega);
            }
        }
        return n;
    }
    size_t lo = (size_t)1 << sparse_degree;
    size_t hi = (size_t)1 << (log_n - sparse_degree - (with_last_level ? 0 : 1));
    if (out) {
        u64 w[4], hw[4];
        cpy4(w, FR->one);
        for (size_t i = 0; i < lo; i++) {
            cpy4(out + 4 * i, w);
            fmul(FR, w, w, omega);
        }
        fpow_u64(FR, hw, omega, lo);
        cpy4(w, FR->one);
        for (size_t i = 0; i < hi; i++) {
            cpy4(out + 4 * (lo + i), w);
            fmul(FR, w, w, hw);
        }
    }
    return lo + hi;
}

int zko_omega(u64 out[4], uint32_t log_n) {
    if (log_n > 28) return -1;
    u64 w[4];
    fmul(FR, w, FR_ROOT_CANON, FR->r2); /* to Montgomery */
    for (uint32_t i = log_n; i < 28; i++) fsqr(FR, w, w);
    cpy4(out, w);
    return 0;
}

int zko_naive_dft(u64 *out, const u64 *a, size_t n, const u64 omega[4]) {
#pragma omp parallel for schedule(dynamic, 4)
    for (size_t k = 0; k < n; k++) {
        u64 wk[4], w[4], acc[4] = {0, 0, 0, 0}, t[4];
        fpow_u64(FR, wk, omega, k);
        cpy4(w, FR->one);
        for (size_t i = 0; i < n; i++) {
            fmul(FR, t, a + 4 * i, w);
            fadd(FR, acc, acc, t);
            fmul(FR, w, w, wk);
        }
        cpy4(out + 4 * k, acc);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* G1: Jacobian arithmetic over Fq, a = 0, b = 3                              */
/* (formulas: dbl-2009-l, madd-2007-bl, add-2007-bl from the EFD)            */
/* ------------------------------------------------------------------------ */
typedef struct { u64 x[4], y[4], z[4]; } jac_t;
typedef struct { u64 x[4], y[4]; } aff_t;

static inline int jac_is_inf(const jac_t *p) { return is_zero4(p->z); }
static inline void jac_set_inf(jac_t *p) { memset(p, 0, sizeof(*p)); }
static inline int aff_is_inf(const aff_t *p) { return is_zero4(p->x) && is_zero4(p->y); }

static void jac_dbl(jac_t *r, const jac_t *p) {
    if (jac_is_inf(p) || is_zero4(p->y)) {
        jac_set_inf(r);
        return;
    }
    u64 A[4], B[4], C[4], D[4], E[4], F[4], t[4], x3[4], y3[4], z3[4];
    fsqr(FQ, A, p->x);
    fsqr(FQ, B, p->y);
    fsqr(FQ, C, B);
    fadd(FQ, t, p->x, B);
    fsqr(FQ, t, t);
    fsub(FQ, t, t, A);
    fsub(FQ, t, t, C);
    fdbl(FQ, D, t);
    fdbl(FQ, E, A);
    fadd(FQ, E, E, A);
    fsqr(FQ, F, E);
    fdbl(FQ, t, D);
    fsub(FQ, x3, F, t);
    fsub(FQ, t, D, x3);
    fmul(FQ, y3, E, t);
    fdbl(FQ, C, C);
    fdbl(FQ, C, C);
    fdbl(FQ, C, C);
    fsub(FQ, y3, y3, C);
    fmul(FQ, z3, p->y, p->z);
    fdbl(FQ, z3, z3);
    cpy4(r->x, x3);
    cpy4(r->y, y3);
    cpy4(r->z, z3);
}

static void jac_add_aff(jac_t *r, const jac_t *p, const aff_t *q) {
    if (aff_is_inf(q)) {
        if (r != p) *r = *p;
        return;
    }
    if (jac_is_inf(p)) {
        cpy4(r->x, q->x);
        cpy4(r->y, q->y);
        cpy4(r->z, FQ->one);
        return;
    }
    u64 Z1Z1[4], U2[4], S2[4], H[4], HH[4], I[4], J[4], rr[4], V[4], t[4];
    fsqr(FQ, Z1Z1, p->z);
    fmul(FQ, U2, q->x, Z1Z1);
    fmul(FQ, S2, q->y, p->z);
    fmul(FQ, S2, S2, Z1Z1);
    fsub(FQ, H, U2, p->x);
    fsub(FQ, rr, S2, p->y);
    if (is_zero4(H)) {
        if (is_zero4(rr)) {
            jac_dbl(r, p);
        } else {
            jac_set_inf(r);
        }
        return;
    }
    fdbl(FQ, rr, rr);
    fsqr(FQ, HH, H);
    fdbl(FQ, I, HH);
    fdbl(FQ, I, I);
    fmul(FQ, J, H, I);
    fmul(FQ, V, p->x, I);
    jac_t o;
    fsqr(FQ, o.x, rr);
    fsub(FQ, o.x, o.x, J);
    fsub(FQ, o.x, o.x, V);
    fsub(FQ, o.x, o.x, V);
    fsub(FQ, t, V, o.x);
    fmul(FQ, o.y, rr, t);
    fmul(FQ, t, p->y, J);
    fdbl(FQ, t, t);
    fsub(FQ, o.y, o.y, t);
    fadd(FQ, o.z, p->z, H);
    fsqr(FQ, o.z, o.z);
    fsub(FQ, o.z, o.z, Z1Z1);
    fsub(FQ, o.z, o.z, HH);
    *r = o;
}

static void jac_add(jac_t *r, const jac_t *p, const jac_t *q) {
    if (jac_is_inf(q)) {
        if (r != p) *r = *p;
        return;
    }
    if (jac_is_inf(p)) {
        if (r != q) *r = *q;
        return;
    }
    u64 Z1Z1[4], Z2Z2[4], U1[4], U2[4], S1[4], S2[4], H[4], I[4], J[4], rr[4], V[4], t[4];
    fsqr(FQ, Z1Z1, p->z);
    fsqr(FQ, Z2Z2, q->z);
    fmul(FQ, U1, p->x, Z2Z2);
    fmul(FQ, U2, q->x, Z1Z1);
    fmul(FQ, S1, p->y, q->z);
    fmul(FQ, S1, S1, Z2Z2);
    fmul(FQ, S2, q->y, p->z);
    fmul(FQ, S2, S2, Z1Z1);
    fsub(FQ, H, U2, U1);
    fsub(FQ, rr, S2, S1);
    if (is_zero4(H)) {
        if (is_zero4(rr)) {
            jac_dbl(r, p);
        } else {
            jac_set_inf(r);
        }
        return;
    }
    fdbl(FQ, rr, rr);
    fdbl(FQ, I, H);
    fsqr(FQ, I, I);
    fmul(FQ, J, H, I);
    fmul(FQ, V, U1, I);
    jac_t o;
    fsqr(FQ, o.x, rr);
    fsub(FQ, o.x, o.x, J);
    fsub(FQ, o.x, o.x, V);
    fsub(FQ, o.x, o.x, V);
    fsub(FQ, t, V, o.x);
    fmul(FQ, o.y, rr, t);
    fmul(FQ, t, S1, J);
    fdbl(FQ, t, t);
    fsub(FQ, o.y, o.y, t);
    fadd(FQ, o.z, p->z, q->z);
    fsqr(FQ, o.z, o.z);
    fsub(FQ, o.z, o.z, Z1Z1);
    fsub(FQ, o.z, o.z, Z2Z2);
    fmul(FQ, o.z, o.z, H);
    *r = o;
}

static void jac_to_aff(aff_t *r, const jac_t *p) {
    if (jac_is_inf(p)) {
        memset(r, 0, sizeof(*r));
        return;
    }
    u64 zi[4], zi2[4], zi3[4];
    finv(FQ, zi, p->z);
    fsqr(FQ, zi2, zi);
    fmul(FQ, zi3, zi2, zi);
    fmul(FQ, r->x, p->x, zi2);
    fmul(FQ, r->y, p->y, zi3);
}

void zko_g1_normalize(u64 out_xy[8], const u64 jac[12]) {
    jac_t p;
    memcpy(&p, jac, sizeof(p));
    aff_t a;
    jac_to_aff(&a, &p);
    memcpy(out_xy, &a, sizeof(a));
}

int zko_g1_on_curve(const u64 xy[8]) {
    aff_t a;
    memcpy(&a, xy, sizeof(a));
    if (aff_is_inf(&a)) return 1;
    if (geq4(a.x, FQ->p) || geq4(a.y, FQ->p)) return 0;
    u64 y2[4], x3[4], b[4], three[4] = {3, 0, 0, 0};
    fsqr(FQ, y2, a.y);
    fsqr(FQ, x3, a.x);
    fmul(FQ, x3, x3, a.x);
    fmul(FQ, b, three, FQ->r2);
    fadd(FQ, x3, x3, b);
    return eq4(x3, y2);
}

/* scalar given in Montgomery form; multiplies by its canonical value */
static void jac_scalar_mul(jac_t *r, const aff_t *base, const u64 k_mont[4]) {
    u64 k[4];
    zko_from_mont(0, k, k_mont);
    jac_t acc;
    jac_set_inf(&acc);
    for (int i = 3; i >= 0; i--)
        for (int b = 63; b >= 0; b--) {
            jac_dbl(&acc, &acc);
            if ((k[i] >> b) & 1) jac_add_aff(&acc, &acc, base);
        }
    *r = acc;
}

void zko_g1_scalar_mul(u64 out_xy[8], const u64 base_xy[8], const u64 scalar_mont[4]) {
    aff_t b;
    memcpy(&b, base_xy, sizeof(b));
    jac_t r;
    jac_scalar_mul(&r, &b, scalar_mont);
    aff_t a;
    jac_to_aff(&a, &r);
    memcpy(out_xy, &a, sizeof(a));
}

void zko_g1_add_affine(u64 out_xy[8], const u64 a_xy[8], const u64 b_xy[8]) {
    jac_t p;
    aff_t a, b;
    memcpy(&a, a_xy, sizeof(a));
    memcpy(&b, b_xy, sizeof(b));
    jac_set_inf(&p);
    jac_add_aff(&p, &p, &a);
    jac_add_aff(&p, &p, &b);
    jac_to_aff(&a, &p);
    memcpy(out_xy, &a, sizeof(a));
}

/* generator (1, 2) in Montgomery form */
static void g1_generator(aff_t *g) {
    u64 one[4] = {1, 0, 0, 0}, two[4] = {2, 0, 0, 0};
    fmul(FQ, g->x, one, FQ->r2);
    fmul(FQ, g->y, two, FQ->r2);
}

/* fixed-base table T[w][d] = [d * 16^w] G, w < 64, d in 1..15, affine */
static aff_t *g_table = NULL;
static void build_gen_table(void) {
#pragma omp critical(zko_gen_table)
    if (!g_table) {
        aff_t *t = (aff_t *)malloc(sizeof(aff_t) * 64 * 16);
        aff_t g;
        g1_generator(&g);
        jac_t base, cur;
        jac_set_inf(&base);
        jac_add_aff(&base, &base, &g);
        for (int w = 0; w < 64; w++) {
            memset(&t[w * 16], 0, sizeof(aff_t));
            cur = base;
            for (int d = 1; d < 16; d++) {
                jac_to_aff(&t[w * 16 + d], &cur);
                jac_add(&cur, &cur, &base);
            }
            for (int s = 0; s < 4; s++) jac_dbl(&base, &base);
        }
        g_table = t;
    }
}

void zko_rand_bases(u64 *bases_xy, u64 *k_mont, size_t n, u64 seed, size_t start, int threads) {
    build_gen_table();
    const size_t CH = 256;
#pragma omp parallel for num_threads(nthreads(threads)) schedule(dynamic, 1)
    for (size_t s = 0; s < n; s += CH) {
        size_t e = s + CH < n ? s + CH : n;
        size_t m = e - s;
        jac_t pts[256];
        u64 prod[256][4];
        for (size_t i = 0; i < m; i++) {
            u64 km[4], kc[4];
            rand_below_r(km, seed ^ 0xba5e5ba5e5ULL, start + s + i);
            if (is_zero4(km)) km[0] = 1; /* never the identity */
            if (k_mont) cpy4(k_mont + 4 * (s + i), km);
            zko_from_mont(0, kc, km);
            jac_t acc;
            jac_set_inf(&acc);
            for (int w = 0; w < 64; w++) {
                int d = (int)((kc[w / 16] >> (4 * (w % 16))) & 15);
                if (d) jac_add_aff(&acc, &acc, &g_table[w * 16 + d]);
            }
            pts[i] = acc;
        }
        /* batch normalisation (Montgomery's trick) */
        u64 acc[4];
        cpy4(acc, FQ->one);
        for (size_t i = 0; i < m; i++) {
            cpy4(prod[i], acc);
            fmul(FQ, acc, acc, pts[i].z);
        }
        u64 inv[4];
        finv(FQ, inv, acc);
        for (size_t i = m; i-- > 0;) {
            u64 zi[4], zi2[4], zi3[4];
            fmul(FQ, zi, inv, prod[i]);
            fmul(FQ, inv, inv, pts[i].z);
            fsqr(FQ, zi2, zi);
            fmul(FQ, zi3, zi2, zi);
            fmul(FQ, bases_xy + 8 * (s + i), pts[i].x, zi2);
            fmul(FQ, bases_xy + 8 * (s + i) + 4, pts[i].y, zi3);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* MSM: halo2 best_multiexp / multiexp_serial                                */
/* ------------------------------------------------------------------------ */
/* c-bit window `segment` of a canonical scalar (halo2 get_at, curve.cuh:108-130) */
static inline unsigned get_at(unsigned segment, unsigned c, const u64 k[4]) {
    unsigned skip = segment * c;
    if (skip >= 256) return 0;
    unsigned w = skip / 64, b = skip % 64;
    u64 v = k[w] >> b;
    if (b + c > 64 && w + 1 < 4) v |= k[w + 1] << (64 - b);
    return (unsigned)(v & ((1ULL << c) - 1));
}

typedef struct {
    int kind; /* 0 none, 1 affine, 2 jacobian */
    aff_t a;
    jac_t j;
} bucket_t;

static void multiexp_serial(jac_t *acc, const u64 *scalars_mont, const aff_t *bases, size_t n) {
    unsigned c;
    if (n < 4)
        c = 1;
    else if (n < 32)
        c = 3;
    else
        c = (unsigned)ceil(log((double)n)); /* halo2: (n as f64).ln().ceil() */
    u64 *canon = (u64 *)malloc(sizeof(u64) * 4 * (n ? n : 1));
    for (size_t i = 0; i < n; i++) zko_from_mont(0, canon + 4 * i, scalars_mont + 4 * i);
    size_t nb = ((size_t)1 << c) - 1;
    bucket_t *bk = (bucket_t *)malloc(sizeof(bucket_t) * nb);
    unsigned segments = 256 / c + 1;
    for (int seg = (int)segments - 1; seg >= 0; seg--) {
        for (unsigned d = 0; d < c; d++) jac_dbl(acc, acc);
        for (size_t b = 0; b < nb; b++) bk[b].kind = 0;
        for (size_t i = 0; i < n; i++) {
            unsigned co = get_at((unsigned)seg, c, canon + 4 * i);
            if (!co) continue;
            bucket_t *B = &bk[co - 1];
            if (B->kind == 0) {
                B->a = bases[i];
                B->kind = 1;
            } else if (B->kind == 1) {
                jac_set_inf(&B->j);
                jac_add_aff(&B->j, &B->j, &B->a);
                jac_add_aff(&B->j, &B->j, &bases[i]);
                B->kind = 2;
            } else {
                jac_add_aff(&B->j, &B->j, &bases[i]);
            }
        }
        jac_t running;
        jac_set_inf(&running);
        for (size_t b = nb; b-- > 0;) {
            if (bk[b].kind == 1)
                jac_add_aff(&running, &running, &bk[b].a);
            else if (bk[b].kind == 2)
                jac_add(&running, &running, &bk[b].j);
            jac_add(acc, acc, &running);
        }
    }
    free(bk);
    free(canon);
}

int zko_multiexp(u64 out_xy[8], const u64 *scalars_mont, const u64 *bases_xy, size_t n, int threads) {
    int T = nthreads(threads);
    const aff_t *bases = (const aff_t *)bases_xy;
    jac_t total;
    jac_set_inf(&total);
    if (n > (size_t)T) {
        size_t chunk = n / T;
        size_t nchunks = (n + chunk - 1) / chunk;
        jac_t *res = (jac_t *)calloc(nchunks, sizeof(jac_t));
#pragma omp parallel for num_threads(T) schedule(dynamic, 1)
        for (size_t ci = 0; ci < nchunks; ci++) {
            size_t s = ci * chunk, e = s + chunk < n ? s + chunk : n;
            jac_set_inf(&res[ci]);
            multiexp_serial(&res[ci], scalars_mont + 4 * s, bases + s, e - s);
        }
        for (size_t ci = 0; ci < nchunks; ci++) jac_add(&total, &total, &res[ci]);
        free(res);
    } else {
        multiexp_serial(&total, scalars_mont, bases, n);
    }
    aff_t a;
    jac_to_aff(&a, &total);
    memcpy(out_xy, &a, sizeof(a));
    return 0;
}

int zko_naive_msm(u64 out_xy[8], const u64 *scalars_mont, const u64 *bases_xy, size_t n) {
    jac_t total, t;
    jac_set_inf(&total);
    for (size_t i = 0; i < n; i++) {
        aff_t b;
        memcpy(&b, bases_xy + 8 * i, sizeof(b));
        jac_scalar_mul(&t, &b, scalars_mont + 4 * i);
        jac_add(&total, &total, &t);
    }
    aff_t a;
    jac_to_aff(&a, &total);
    memcpy(out_xy, &a, sizeof(a));
    return 0;
}
