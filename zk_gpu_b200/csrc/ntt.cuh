// ntt.cuh — Fr number-theoretic transform on sm_100a: plans, device tables,
// and the launch entry used by the C ABI, the batcher and the LDE pipeline.
//
// Algorithm: a natural-order-in / natural-order-out DFT
//     A[k] = sum_i a[i] * w^(i k)           (w of order exactly n = 2^log_n)
// computed as a mixed-radix four-step over p passes with bit widths
// b_1 .. b_p (sum = log_n, each <= 12).  Pass t views the data as
// [O_t][m_t][J_t] (m_t = 2^b_t, O_t = 2^(b_1+..+b_(t-1)), J_t = 2^(b_(t+1)+..))
// and runs one m_t-point DIF DFT per (o, j) column, then multiplies output
// k of column j by the twist w_(m_t J_t)^(k j) and writes it back in place.
// The last pass writes element (o, k) to rev(o) + (n / m_p) k, where rev
// reverses o's mixed-radix digits, which lands every A[k] at index k.
// This replaces the reference's four-step 1024 x n/1024 path
// (cuda/fft.cu:61-156, 275-405): one kernel per pass instead of five,
// every thread busy, twiddles from device tables instead of pow_vartime.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstddef>
#include <memory>

#include "field.cuh"
#include "host_field.hpp"

namespace zk {

constexpr int NTT_MAX_LOG = 28;   // Fr two-adicity
constexpr int NTT_MAX_PASS = 4;

struct NttPlan {
  int log_n = 0;
  int npass = 0;
  int bits[NTT_MAX_PASS] = {0, 0, 0, 0};
};
NttPlan make_ntt_plan(int log_n);
// Supported plans: log_n <= 2 direct (no passes); one pass of log_n <= 11
// bits; or 2..4 passes of 3..11 bits summing to log_n.
bool ntt_plan_valid(const NttPlan& p);
// The plan the autotuner chose for (device, log_n), else make_ntt_plan.
NttPlan tuned_ntt_plan(int device, int log_n);

// Device tables for one (omega, log_n): per pass the inner roots
// w_m^e (e < m/2) and, for non-final passes, the twist table [k * J + j].
struct NttTables {
  NttPlan plan;
  host::Fr omega;
  fe* inner[NTT_MAX_PASS] = {nullptr, nullptr, nullptr, nullptr};
  fe* twist[NTT_MAX_PASS] = {nullptr, nullptr, nullptr, nullptr};
  size_t bytes = 0;
};

// Coset pre-multiplication: input element x is multiplied by c^x, read as
// lo[x & (2^shift - 1)] * hi[x >> shift].
struct PowTables {
  fe* lo = nullptr;
  fe* hi = nullptr;
  uint32_t shift = 0;
};

// Cached tables for (device, omega, log_n) under the device's current plan;
// thread-safe.  Returns null and sets *err on failure.  The reference keeps
// the tables alive: work that reads them (an enqueued transform, a batch
// graph, a serving wave) holds it until the work is done or destroyed.  The
// cache is capped per device (ZKGPU_TABLE_CACHE_MB, default 8192) and evicts
// its least recently used entries; an evicted table is freed when its last
// holder lets go (cudaFree, which waits for the device).
using NttTablesRef = std::shared_ptr<const NttTables>;
NttTablesRef ntt_tables_get(int device, const host::Fr& omega, int log_n, cudaStream_t s, cudaError_t* err);
// Uncached tables for an explicit plan (the autotuner's trials); free with
// ntt_tables_release after the work using them has finished.
cudaError_t ntt_tables_build(NttTables* t, const NttPlan& plan, const host::Fr& omega, cudaStream_t s);
void ntt_tables_release(NttTables* t);
// Tables for (omega, log_n) written into caller-provided device memory of
// `cap` elements (no allocation); ntt_tables_elems gives the size needed.
size_t ntt_tables_elems(int log_n);
cudaError_t ntt_tables_fill(NttTables* t, const host::Fr& omega, int log_n, fe* mem, size_t cap, cudaStream_t s);
// Two-level power tables for scale * c^x, x < 2^log_n (scale folded into the
// low table; null = 1), allocated from the library pool on `s` (caller frees
// with pow_tables_free on the same stream), or with cudaMalloc when !pooled.
cudaError_t pow_tables_make(PowTables* t, const host::Fr& c, int log_n, cudaStream_t s,
                            const host::Fr* scale = nullptr, bool pooled = true);
void pow_tables_free(PowTables* t, cudaStream_t s);
// Cached (device, c, log_n, scale) power tables, under the same cap and
// lifetime rules as ntt_tables_get.
using PowTablesRef = std::shared_ptr<const PowTables>;
PowTablesRef pow_tables_get(int device, const host::Fr& c, int log_n, cudaStream_t s, cudaError_t* err,
                            const host::Fr* scale = nullptr);
// Bytes the device's table caches hold, and dropping every cached entry
// (entries still held by work stay alive until it lets go).
uint64_t table_cache_bytes(int device);
uint64_t table_cache_builds(int device);  // tables built so far on `device` (cache misses)
void table_cache_clear(int device);

// Parameters of one pass launch (kernel argument / batch descriptor).
struct PassParams {
  const fe* in;
  fe* out;
  const fe* inner;   // w_m^e, e < m/2 (R' form)
  const fe* twist;   // [k * J + j], non-final passes (R' form)
  const fe* pre_lo;  // coset powers (first pass), or null
  const fe* pre_hi;
  uint32_t pre_shift;
  uint32_t log_J;
  uint32_t log_O;
  uint32_t log_m1;
  uint32_t nprev;
  uint32_t prev_bits[NTT_MAX_PASS];
  uint32_t G;
  uint32_t is_final;
  uint32_t has_post;
  fe post;  // R' form
  // final pass: output k multiplied by post_lo[k & mask] * post_hi[k >> shift]
  const fe* post_lo;
  const fe* post_hi;
  uint32_t post_shift;
  // first pass: rows >= in_rows are known zeros (zero-padded input), 0 = all
  uint32_t in_rows;
};

// Optional work fused into a transform.
struct NttFuse {
  const PowTables* pre = nullptr;       // input i times c^i
  const host::Fr* post = nullptr;       // every output times a constant
  const PowTables* post_tab = nullptr;  // output k times the table's k-th power
  uint64_t nonzero = 0;                 // only inputs [0, nonzero) may be non-zero (0 = all)
  const fe* src = nullptr;              // read the input from here instead of d_a (d_a gets the result)
};

// Pass k of the plan in `t` over d_a / d_tmp; returns its CTA count.
uint64_t ntt_pass_params(const NttTables& t, int k, fe* d_a, fe* d_tmp, const PowTables* pre, const host::Fr* post,
                         PassParams* pp);
uint64_t ntt_pass_params(const NttTables& t, int k, fe* d_a, fe* d_tmp, const NttFuse& f, PassParams* pp);

// One pass of one transform inside a batch launch.
struct BatchPass {
  PassParams p;
  uint32_t B;
  uint32_t ntiles;
  uint32_t tile_base;  // global index of this pass's first tile
  uint32_t dep;        // index of the pass this one waits for, or ~0u
  uint32_t dep_tiles;  // tiles of that pass
};
// Launch the persistent batch kernel over `npass` descriptors (device memory,
// ordered by level), with counters next/done/err zeroed by the caller.
// Every dependency wait gives up after spin_cycles SM clocks (default about
// two seconds at the B200 boost clock), sets *d_err and stops the kernel.
constexpr uint64_t NTT_BATCH_SPIN_CYCLES = 4000000000ull;
cudaError_t ntt_batch_launch(const BatchPass* d_passes, uint32_t npass, uint32_t total_tiles, uint32_t* d_next,
                             uint32_t* d_done, uint32_t* d_err, int grid, cudaStream_t s,
                             uint64_t spin_cycles = NTT_BATCH_SPIN_CYCLES);
int ntt_batch_grid(int device);

// Runs the NTT over d_a (2^log_n elements, in place).  d_tmp is scratch of
// the same size (unused for single-pass plans).  pre (nullable) applies the
// coset powers before the transform; post (nullable, host value) scales every
// output; outputs are canonical.
cudaError_t ntt_run(const NttTables& t, fe* d_a, fe* d_tmp, const PowTables* pre, const host::Fr* post,
                    cudaStream_t s);
cudaError_t ntt_run(const NttTables& t, fe* d_a, fe* d_tmp, const NttFuse& f, cudaStream_t s);

// Number of launches ntt_run issues for a plan (for launch accounting).
inline int ntt_launches(const NttPlan& p) { return p.npass; }

// Elementwise helpers used by the LDE pipeline.
cudaError_t fr_scale_copy(fe* dst, const fe* src, size_t n, size_t dst_stride, const PowTables* powc,
                          cudaStream_t s);

}  // namespace zk
