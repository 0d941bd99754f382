/*
 * zkgpu.h — C ABI of libzkgpu.so, the B200 (sm_100a) implementation of the
 * halo2/BN256 prover hot path: the Fr NTT (forward, inverse, coset /
 * extended-domain LDE) and the G1 Pippenger MSM.
 *
 * Data layout (all entry points): one field element = 4 x uint64_t little
 * endian limbs in Montgomery form (R = 2^256), canonical (< modulus) — the
 * layout of the reference's BigNum (cuda/bn256.h:10-13) and of halo2curves'
 * Fr / Fq.  Affine points are {x, y} with the identity encoded as (0, 0);
 * projective points are Jacobian {X, Y, Z} (x = X/Z^2, y = Y/Z^3) with the
 * identity Z = 0 (cuda/bn256.h:15-28, src/lib.rs:22-35).
 *
 * Status convention: 0 = success, otherwise a ZKGPU_E* code below.  No entry
 * point prints, exits or aborts the host process (the reference exit()s on
 * CUDA errors, cuda/fft.cu:380-395).
 */
#ifndef ZKGPU_H
#define ZKGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/lib.rs:22-28 (#[repr(C)] GpuAffine) */
typedef struct {
    uint64_t x[4];
    uint64_t y[4];
} GpuAffine;

/* src/lib.rs:30-35 (#[repr(C)] GpuProjective) */
typedef struct {
    uint64_t x[4];
    uint64_t y[4];
    uint64_t z[4];
} GpuProjective;

enum {
    ZKGPU_OK = 0,
    ZKGPU_EINVAL = 1,    /* bad size, null pointer, omega not of order n, ... */
    ZKGPU_ENOMEM = 2,    /* device allocation failed */
    ZKGPU_ECUDA = 3,     /* CUDA runtime error (message: zkgpu_last_error) */
    ZKGPU_ETIMEOUT = 4,  /* a bounded device wait expired */
    ZKGPU_EADMIT = 5,    /* serving: job larger than the HBM budget */
    ZKGPU_ENODEV = 6,    /* no such CUDA device */
    ZKGPU_EBUSY = 7      /* serving: queue full / shut down */
};

/* ======================================================================
 * Reference-compatible entry points.  Signatures are the Rust declarations
 * of src/api.rs:3-14 (usize -> size_t, u64 -> uint64_t); they are
 * synchronous and operate on caller-owned HOST buffers, like the C
 * definitions they replace (cuda/fft.cu:553-583).
 * ====================================================================== */

/* src/api.rs:4 / cuda/fft.cu:554-558: device self-test.  Runs a field
 * known-answer check on `device_id`; returns 0 on success. */
uint64_t do_fft_ffi(size_t device_id);

/* src/api.rs:6 / cuda/fft.cu:560-564: in-place forward NTT of `req`
 * (n = 2^log_n elements, natural order in and out) with root `omega`.
 * `twiddle` / `twiddle_size` (halo2 generate_twiddle_lookup_table(omega,
 * log_n, 10, true)) are accepted for ABI compatibility; the device derives
 * its own tables from `omega`, which must have order exactly n. */
uint64_t parallel_fft_api(size_t device_id, uint64_t *req, const uint64_t *omega, const uint64_t *twiddle,
                          uint64_t n, uint64_t log_n, uint64_t twiddle_size);

/* src/api.rs:8 / cuda/fft.cu:566-570: in-place inverse NTT: forward NTT
 * with `omega` (the caller passes w^-1) then every element * `divisor`
 * (the caller passes n^-1). */
uint64_t parallel_ifft_api(size_t device_id, uint64_t *req, const uint64_t *omega, const uint64_t *twiddle,
                           uint64_t n, uint64_t log_n, uint64_t twiddle_size, const uint64_t *divisor);

/* src/api.rs:10 / cuda/fft.cu:572-576, :223-232: req[i] *= c^i, then the
 * forward NTT (one part of the extended-domain evaluation). */
uint64_t parallel_coeff_to_extended_part_api(size_t device_id, uint64_t *req, const uint64_t *omega,
                                             const uint64_t *twiddle, uint64_t n, uint64_t log_n,
                                             uint64_t twiddle_size, const uint64_t *c);

/* src/api.rs:12 / cuda/fft.cu:578-582, :450-551: acc = sum_i data[i] *
 * bases[i] (data: Fr Montgomery scalars, bases: affine Fq Montgomery).
 * Any length >= 0 (the reference needs a power of two > 256).  The result
 * is written normalised: Z = Montgomery one, or all-zero for the identity. */
uint64_t parallel_msm_api(size_t device_id, const uint64_t *data, const GpuAffine *bases, uint64_t lenght,
                          GpuProjective *acc);

/* ======================================================================
 * Host-buffer API with short names (fft / ifft / coset_fft / msm).
 * ====================================================================== */
int zkgpu_fft(int device, uint64_t *a, uint32_t log_n, const uint64_t omega[4]);
int zkgpu_ifft(int device, uint64_t *a, uint32_t log_n, const uint64_t omega_inv[4], const uint64_t divisor[4]);
int zkgpu_coset_fft(int device, uint64_t *a, uint32_t log_n, const uint64_t omega[4], const uint64_t c[4]);
int zkgpu_msm(int device, const uint64_t *scalars, const uint64_t *bases_xy, uint64_t n, uint64_t out_xyz[12]);

/* halo2 coset LDE as one call (lagrange -> extended):
 *   coeffs = ifft(values, omega_inv, n^-1);  coeffs[i] *= g^i;
 *   ext    = fft(zero-pad(coeffs, 2^log_ext), omega_ext)      (natural order)
 * values: 2^log_n host elements (read only); ext: 2^log_ext host elements. */
int zkgpu_lagrange_to_extended(int device, const uint64_t *values, uint32_t log_n, uint64_t *ext, uint32_t log_ext,
                               const uint64_t omega_inv[4], const uint64_t divisor[4], const uint64_t g[4],
                               const uint64_t omega_ext[4]);
/* The inverse step, halo2 extended -> coefficients (the quotient polynomial's
 * path back from the extended domain):
 *   a = ifft(ext, omega_ext_inv, ext_divisor = 2^-log_ext);  a[i] *= g_inv^i;
 *   out = a[0, m)                                             (truncate, m <= 2^log_ext)
 * ext: 2^log_ext host elements (read only); out: m host elements. */
int zkgpu_extended_to_coeff(int device, const uint64_t *ext, uint32_t log_ext, uint64_t *out, uint64_t m,
                            const uint64_t omega_ext_inv[4], const uint64_t ext_divisor[4], const uint64_t g_inv[4]);

/* ======================================================================
 * Device-resident API: pointers are device memory on `device`, work is
 * enqueued on `stream` (a cudaStream_t, NULL = legacy default) and the call
 * returns without synchronising.  Scratch comes from the stream's pool.
 * ====================================================================== */
/* in place; optional coset (a[i] *= c^i first) and post scale (every output * scale) */
int zkgpu_ntt_dev(int device, uint64_t *d_a, uint32_t log_n, const uint64_t omega[4], const uint64_t *coset_c,
                  const uint64_t *post_scale, void *stream);
/* d_values (2^log_n) -> d_ext (2^log_ext), the same pipeline as
 * zkgpu_lagrange_to_extended; d_values is not modified. */
int zkgpu_lagrange_to_extended_dev(int device, const uint64_t *d_values, uint32_t log_n, uint64_t *d_ext,
                                   uint32_t log_ext, const uint64_t omega_inv[4], const uint64_t divisor[4],
                                   const uint64_t g[4], const uint64_t omega_ext[4], void *stream);
int zkgpu_extended_to_coeff_dev(int device, const uint64_t *d_ext, uint32_t log_ext, uint64_t *d_out, uint64_t m,
                                const uint64_t omega_ext_inv[4], const uint64_t ext_divisor[4], const uint64_t g_inv[4],
                                void *stream);
/* No counterpart in the reference.  The same in-place NTT as zkgpu_ntt_dev
 * (no coset, no scale) for callers that cannot allocate device memory — code
 * running under stream capture, or inside a runtime that owns every device
 * allocation.  It calls no allocator: its scratch (ping-pong buffer and root
 * tables) is a static device array in the library sized for log_n <=
 * ZKGPU_STATIC_NTT_MAX_LOG (about 16.8 MB per GPU, held until process exit);
 * larger log_n returns ZKGPU_EINVAL.  It always runs the built-in pass plan
 * for log_n (the autotuner's choices are not consulted; results are the same,
 * only the speed can differ).  The first call on a device resolves the
 * array's address, so make it before any stream capture starts.  All calls on
 * a device share the array: calls whose work overlaps on the GPU race and
 * must be serialised by the caller (one stream or events). */
#define ZKGPU_STATIC_NTT_MAX_LOG 18
int zkgpu_ntt_dev_static(int device, uint64_t *d_a, uint32_t log_n, const uint64_t omega[4], void *stream);
/* Element-wise ops on device vectors of n Fr elements (extended-domain
 * evaluations in halo2's quotient step: gates combined as h = h * y + e,
 * polynomial products and sums).  No counterpart in the reference, whose
 * only element-wise device op is distribute_powers (cuda/fft.cu:223-232);
 * the operations restate halo2's Polynomial Mul / Add / Sub / scalar Mul on
 * ExtendedLagrangeCoeff vectors.  d_out may alias d_a or d_b. */
#define ZKGPU_EW_MUL 0u   /* out[i] = a[i] * b[i] */
#define ZKGPU_EW_ADD 1u   /* out[i] = a[i] + b[i] */
#define ZKGPU_EW_SUB 2u   /* out[i] = a[i] - b[i] */
#define ZKGPU_EW_SCALE 3u /* out[i] = a[i] * c            (d_b unused) */
#define ZKGPU_EW_AXPY 4u  /* out[i] = a[i] * c + b[i] */
int zkgpu_ew_dev(int device, uint32_t op, uint64_t *d_out, const uint64_t *d_a, const uint64_t *d_b,
                 const uint64_t c[4], uint64_t n, void *stream);
/* halo2 EvaluationDomain::divide_by_vanishing_poly on device: d_ext holds the
 * 2^log_ext evaluations on the coset g * <omega_ext>; element k is divided by
 * t(X) = X^n - 1 there, t_k = g^n omega_ext^(n k) - 1, which takes only
 * 2^(log_ext - log_n) <= 64 distinct values (inverted once on the host).
 * ZKGPU_EINVAL when t vanishes somewhere on the coset. */
int zkgpu_divide_by_vanishing_dev(int device, uint64_t *d_ext, uint32_t log_n, uint32_t log_ext, const uint64_t g[4],
                                  const uint64_t omega_ext[4], void *stream);
/* d_out_xyz receives the Jacobian sum (12 words, device memory), normalised
 * (Z = Montgomery one, or all zero for the identity); the call stays
 * asynchronous on `stream` (its last, serial step runs on the host as a
 * stream-ordered host function). */
int zkgpu_msm_dev(int device, const uint64_t *d_scalars, const uint64_t *d_bases_xy, uint64_t n, uint64_t *d_out_xyz,
                  void *stream);
/* d_out_xy[i] = k_i * base (affine, Fq Montgomery, (0, 0) for the identity),
 * k_i = d_scalars[i] (Fr Montgomery); base_xy is a host value.  Generates MSM
 * bases as multiples of a fixed point, e.g. of the generator (1, 2).
 * Synchronous on `stream`. */
int zkgpu_g1_mul_fixed_dev(int device, const uint64_t base_xy[8], const uint64_t *d_scalars, uint64_t n,
                           uint64_t *d_out_xy, void *stream);

/* ======================================================================
 * Batched NTTs: many transforms of uneven sizes in one persistent launch,
 * replayed from a CUDA graph.  Replaces the per-job device choice and
 * one-call-per-job flow of src/gpulock.rs:133-226 + cuda/fft.cu:275-405.
 * ====================================================================== */
#define ZKGPU_JOB_COSET 1u /* multiply element i by coset^i before the transform */
#define ZKGPU_JOB_SCALE 2u /* multiply every output by scale (e.g. n^-1 for an inverse) */
typedef struct {
    uint64_t *data;     /* device memory, 2^log_n elements, transformed in place */
    uint32_t log_n;     /* 3 .. 28 */
    uint32_t flags;     /* ZKGPU_JOB_* */
    uint64_t omega[4];  /* root of order exactly 2^log_n (w^-1 for an inverse) */
    uint64_t coset[4];
    uint64_t scale[4];
} zkgpu_ntt_job;
/* Build a batch (tables, scratch, work list, graph).  The jobs' data
 * pointers are baked in: refill the same buffers and run again. */
int zkgpu_ntt_batch_create(int device, const zkgpu_ntt_job *jobs, uint32_t njobs, void **handle);
/* Enqueue one run on `stream` (graph launch); one run at a time per handle. */
int zkgpu_ntt_batch_run(void *handle, void *stream);
/* After a run completed: ZKGPU_ETIMEOUT if a bounded dependency wait expired. */
int zkgpu_ntt_batch_check(void *handle);
void zkgpu_ntt_batch_info(void *handle, uint32_t *passes, uint32_t *tiles, int *grid);
void zkgpu_ntt_batch_destroy(void *handle);

/* ======================================================================
 * Autotuner: per device and size, the NTT plan (pass widths b_k, 3..11 bits;
 * each pass runs radix-2^b_k columns in CTA tiles of 2^b_k x G elements,
 * G = 2^(11 - b_k)) and the MSM window width c, picked by timing candidates
 * on the device.  Replaces the fixed 1024 x n/1024 split of
 * cuda/fft.cu:275-405 and the ceil(ln len) window of cuda/fft.cu:165-172.
 * Choices change speed only: every plan and window is bit-exact.  Installed
 * choices apply to later calls on that device (tables of a new plan are built
 * on first use).
 * ====================================================================== */
#define ZKGPU_TUNE_NTT 1u         /* time one transform per size */
#define ZKGPU_TUNE_MSM 2u         /* time MSMs of 2^log_n points */
#define ZKGPU_TUNE_NTT_BATCHED 4u /* time batches of transforms of each size (the batcher's case) */
/* Tune sizes 2^log_min .. 2^log_max; reps timed runs per candidate (0 = 3);
 * *ms_spent (nullable) receives the device time the tuning took. */
int zkgpu_autotune(int device, uint32_t what, uint32_t log_min, uint32_t log_max, uint32_t reps, double *ms_spent);
/* Install a plan (npass = 0: back to the built-in plan for log_n > 2) /
 * read the plan used for (device, log_n).  EINVAL for unsupported plans. */
int zkgpu_tune_set_ntt_plan(int device, uint32_t log_n, uint32_t npass, const uint32_t bits[4]);
int zkgpu_tune_get_ntt_plan(int device, uint32_t log_n, uint32_t *npass, uint32_t bits[4]);
/* Install (c = 0: clear) / read the MSM window for 2^log_n points. */
int zkgpu_tune_set_msm_window(int device, uint32_t log_n, uint32_t c);
int zkgpu_tune_get_msm_window(int device, uint32_t log_n, uint32_t *c);
/* Persist the device's installed choices; load installs the entries recorded
 * for a device of the same name and SM count (*loaded = entries installed). */
int zkgpu_tune_save(int device, const char *path);
int zkgpu_tune_load(int device, const char *path, uint32_t *loaded);

/* ======================================================================
 * Serving loop: continuous batching with HBM-budget admission.  Replaces the
 * reference's GpuLock / get_gpu / THREAD_POOL scheduling
 * (src/gpulock.rs:72-246, src/config.rs:97-127, src/threadpool.rs:34-121).
 * Jobs arrive with host input/output buffers (pinned memory keeps every copy
 * asynchronous); admitted NTT/LDE jobs of one scheduling wave run as one
 * persistent batch launch, MSMs run against resident bases.
 * ====================================================================== */
#define ZKGPU_KIND_NTT 0u /* in place on `output` (input copied from `input`) */
#define ZKGPU_KIND_LDE 1u /* lagrange 2^log_n -> coset extended 2^log_ext */
#define ZKGPU_KIND_MSM 2u /* sum scalars[i] * bases[i], i < n, over a resident base set */
typedef struct {
    uint32_t kind;
    uint32_t log_n;      /* NTT / LDE input size */
    uint32_t log_ext;    /* LDE only */
    uint32_t flags;      /* NTT: ZKGPU_JOB_COSET / ZKGPU_JOB_SCALE */
    uint64_t n;          /* MSM: points */
    uint32_t bases_id;   /* MSM: id from zkgpu_server_add_bases */
    uint32_t reserved;
    const uint64_t *input;  /* NTT/LDE: 2^log_n elements; MSM: n scalars */
    uint64_t *output;       /* NTT: 2^log_n; LDE: 2^log_ext; MSM: 12 words (normalised Jacobian) */
    uint64_t omega[4];      /* NTT: root; LDE: omega_inv of the 2^log_n domain */
    uint64_t coset[4];      /* NTT: coset c; LDE: coset generator g */
    uint64_t scale[4];      /* NTT: output scale; LDE: divisor n^-1 */
    uint64_t omega_ext[4];  /* LDE: root of the 2^log_ext domain */
} zkgpu_job;

typedef struct {
    uint64_t submitted, rejected, completed, failed;
    uint64_t waves, batch_launches;
    uint64_t hbm_budget, hbm_used, hbm_peak;
    uint64_t pending, inflight;
    uint64_t msm_merged_passes; /* multi-MSM passes (MSMs of one wave on shared bases) */
    uint64_t msm_merged_jobs;   /* MSM jobs that ran inside such passes */
    uint64_t table_builds;      /* NTT / coset tables built on this device since the server started (cache misses) */
    uint64_t cache_clears;      /* table caches dropped by the scheduler to make room (nothing in flight) */
    uint64_t memory_waits;      /* admission rounds that waited for a wave to retire (head job did not fit) */
    uint64_t max_launch_us;     /* longest host time the scheduler spent enqueueing one wave */
} zkgpu_server_stats;

/* device memory a job needs while in flight (bytes) */
uint64_t zkgpu_job_footprint(const zkgpu_job *job);
/* Admission policy, simulated on the host (no device): jobs with the given
 * footprints arrive in order; `admit_rounds[i]` receives the scheduling round
 * in which job i is admitted when every admitted job completes one round
 * after admission (-1 = rejected).  Returns the peak bytes in use. */
uint64_t zkgpu_admission_simulate(uint64_t budget, const uint64_t *footprints, uint32_t n, int32_t *admit_rounds);

/* max_wave_jobs: jobs per scheduling wave (0 = 256); up to 8 waves are on
 * the GPU at once.  The server pins 8 x (32 + 8216 x max_wave_jobs) bytes of
 * host memory for its result mailboxes (an MSM job's window sums come back
 * there; 16.8 MB at 256) and 8 x 2048 batch pass descriptors.  At start it
 * takes hbm_budget_bytes (at most the device's free memory less 4 GB) into
 * the library's memory pool, where it stays after zkgpu_server_destroy until
 * zkgpu_release_cached.
 * MSM jobs of one wave against the same bases run as one multi-MSM pass. */
int zkgpu_server_create(int device, uint64_t hbm_budget_bytes, uint32_t max_wave_jobs, void **server);
/* upload a base set once (affine, 8 words per point); it stays resident */
int zkgpu_server_add_bases(void *server, const uint64_t *bases_xy, uint64_t n, uint32_t *bases_id);
/* non-blocking; ZKGPU_EADMIT if the job can never fit the budget */
int zkgpu_server_submit(void *server, const zkgpu_job *job, uint64_t *ticket);
/* wait for a job (timeout_ms 0 = forever); *latency_ms = completion - submit */
int zkgpu_server_wait(void *server, uint64_t ticket, uint32_t timeout_ms, double *latency_ms);
int zkgpu_server_stats_get(void *server, zkgpu_server_stats *out);
void zkgpu_server_destroy(void *server);

/* ======================================================================
 * Diagnostics.
 * ====================================================================== */
/* elementwise field op on host arrays through the device kernels:
 * op 0 = mul, 1 = add, 2 = sub (Montgomery form);  fid 0 = Fr, 1 = Fq;
 * op 3 (Fq only, b unused and may be null) = the inverse of plain canonical
 * integers a < q, 0 for 0: the MSM rounds' divstep inversion */
int zkgpu_field_op(int device, int op, int fid, const uint64_t *a, const uint64_t *b, uint64_t *out, uint64_t n);
/* failure detection: runs a batch whose dependency wait can never be met;
 * the kernel gives up after about spin_us and the call returns
 * ZKGPU_ETIMEOUT (omega12: a root of order 2^12).  No counterpart in the
 * reference, whose scheduler waits without limit (src/gpulock.rs:191-194). */
int zkgpu_selftest_wait_timeout(int device, const uint64_t omega12[4], uint32_t spin_us);
/* Give back the device memory the library keeps cached on `device`: the
 * NTT / coset table caches (capped at ZKGPU_TABLE_CACHE_MB per device,
 * default 8192, least recently used first; a serving loop counts them against
 * its HBM budget) and the unused blocks of the library's own memory pool.
 * Tables still read by live batches or in-flight work stay allocated until
 * that work lets go of them.  No counterpart in the reference, which
 * allocates and frees everything per call (cuda/fft.cu:282-328). */
int zkgpu_release_cached(int device);
/* message of the last ZKGPU_ECUDA on this thread ("" if none) */
const char *zkgpu_last_error(void);
/* kernel launches issued by this thread since the last reset */
uint64_t zkgpu_launch_count(int reset);
/* library version string */
const char *zkgpu_version(void);
/* measured 32-bit integer multiply-add issue rate of `device` (IMAD/s) and
 * the rate of this library's Fr Montgomery product (products/s) */
int zkgpu_int_peak(int device, uint32_t iters, double *imad_per_s, double *modmul_per_s);
/* opt-in CUDA-event timing of each kernel launch, per kernel name */
void zkgpu_prof_enable(int on);
void zkgpu_prof_reset(void);
/* lines "name launches total_ms work_modmul bytes"; returns the line count */
int zkgpu_prof_read(char *buf, uint64_t cap);

#ifdef __cplusplus
}
#endif
#endif /* ZKGPU_H */
