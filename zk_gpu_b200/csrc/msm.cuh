// msm.cuh — G1 multi-scalar multiplication (Pippenger) on sm_100a.
//
//   sum_i s_i * P_i,  s_i in Fr (Montgomery), P_i affine in Fq (Montgomery)
//
// This replaces the reference's one-thread-per-chunk serial Pippenger with
// local-memory buckets (cuda/fft.cu:158-221, 450-551):
//   1. digits   : every scalar -> W signed c-bit digits d_w in
//                 [-2^(c-1), 2^(c-1)]; each non-zero digit is an entry
//                 (bucket = w * 2^(c-1) + |d_w| - 1, point index, sign).
//   2. sort     : counting sort of the entries by bucket (histogram, scan,
//                 scatter), so each bucket's points are contiguous.
//   3. buckets  : pairwise affine additions in rounds, the inverses of each
//                 round from Montgomery's trick (batch-affine accumulation).
//   4. reduce   : per window, sum_b b * B_b by segmented running sums
//                 (segment results T_s + lo_s * S_s), then a block tree sum.
//   5. combine  : Horner over windows, sum_w 2^(c w) W_w, on the host (the
//                 ~250 dependent doublings are serial), normalised Jacobian.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "field.cuh"

namespace zk {

struct MsmPlan {
  int c = 0;         // window bits
  int windows = 0;   // W
  uint32_t buckets = 0;  // per window, 2^(c-1)
  uint32_t seg_len = 0;  // buckets per reduction segment
};
// c_override = 0: the autotuner's window for `device` (-1: the current
// device), else clamp(ceil(log2 n) - 4, 4, 16).
MsmPlan make_msm_plan(uint64_t n, int c_override = 0, int device = -1);
// The window installed by the autotuner for (device, log2 n), or 0.
int tuned_msm_window(int device, int log_n);

// Enqueue the MSM on `s`; d_out receives the Jacobian sum (X, Y, Z: 12 u64,
// normalised to Z = one; all zero for the identity), the last step (Horner
// over the windows) running as a host function on the stream.  Scratch
// comes from the library pool.
// Optional: stop before the last step and leave the per-window sums for the
// host (host::fq::msm_combine_windows), which does the ~250 dependent
// doublings of the Horner step far faster than one GPU thread.
struct MsmWindowsOut {
  fe* d_winsum = nullptr;  // >= plan.windows * 4 elements (XYZZ, R' form)
  uint32_t windows = 0;    // set by msm_run (0 for n = 0)
  uint32_t c = 0;
};
constexpr uint32_t MSM_MAX_WINDOWS = 64;  // c >= 4
// bases_rp: d_bases_xy is already in the R' = 2^260 form of the curve
// arithmetic (msm_convert_bases; resident bases are converted once)
cudaError_t msm_run(const fe* d_scalars, const fe* d_bases_xy, uint64_t n, fe* d_out, cudaStream_t s,
                    int c_override = 0, uint64_t* launches = nullptr, MsmWindowsOut* wout = nullptr,
                    bool bases_rp = false);
// Several MSMs over one base array (the serving loop's jobs against resident
// bases) in one pass: job j's scalars are [off[j], off[j+1]) of d_scalars
// (d_job_off: jobs + 1 offsets in device memory, off[0] = 0), each against
// bases [0, n_j); max_n = the largest n_j.  One window size (the plan of the
// mean job size); job j's window sums land in windows [j W, (j + 1) W) of
// wout->d_winsum (>= jobs * W * 4 elements), W = wout->windows on return.
cudaError_t msm_run_multi(const fe* d_scalars, const fe* d_bases_xy, const uint32_t* d_job_off, uint32_t jobs,
                          uint64_t n_total, uint64_t max_n, cudaStream_t s, uint64_t* launches,
                          MsmWindowsOut* wout, bool bases_rp = false);
// Device scratch one msm_run / msm_run_multi call allocates from the stream
// pool (n_total scalars over `jobs` MSMs; nbases converted unless bases_rp;
// own_winsum: the window sums are not the caller's buffer; the window size of
// `device`, -1 = the current device).
uint64_t msm_scratch_bytes(uint64_t n_total, uint32_t jobs, uint64_t nbases, bool bases_rp, bool own_winsum,
                           int device = -1);
// Affine bases from the API's R form (x 2^256) to the curve arithmetic's
// R' form (x 2^260), canonical; (0, 0) stays (0, 0).  In place is allowed.
cudaError_t msm_convert_bases(const fe* d_in, fe* d_out, uint64_t n, cudaStream_t s);

}  // namespace zk
