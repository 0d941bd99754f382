// msm.cu — Pippenger MSM kernels and orchestration (see msm.cuh).
#include <algorithm>

#include <mutex>
#include <vector>

#include "curve.cuh"
#include "fq_inv.cuh"
#include "host_field.hpp"
#include "msm.cuh"
#include "prof.cuh"
#include "runtime.cuh"

namespace zk {

MsmPlan make_msm_plan(uint64_t n, int c_override, int device) {
  MsmPlan p;
  int lg = 1;
  while ((1ull << lg) < n) lg++;
  int c = lg - 4;
  if (c < 4) c = 4;
  if (c > 16) c = 16;
  if (c_override == 0) {  // the autotuner's choice for this device and size, if any
    int dev = device;
    if (dev >= 0 || cudaGetDevice(&dev) == cudaSuccess) c_override = tuned_msm_window(dev, lg);
  }
  if (c_override >= 3 && c_override <= 20) c = c_override;
  p.c = c;
  p.windows = (254 + c - 1) / c;
  p.buckets = 1u << (c - 1);
  // buckets per reduction segment: a segment thread's latency is its
  // running sum (2L additions); the window kernel then walks B / L segment
  // sums per window, M = B / (256 L) per thread.  Few buckets per window:
  // L = 4 for parallelism; many (2^12 and up): L = 16, which keeps the
  // per-window pass (one block per window) short
  p.seg_len = std::min<uint32_t>(p.buckets >= 4096 ? 16u : 4u, p.buckets);
  return p;
}

// bits [pos, pos + c) of a canonical 256-bit scalar (c <= 20), 0 beyond bit 255
__device__ __forceinline__ uint32_t scalar_bits(const uint32_t s[8], uint32_t pos, uint32_t c) {
  const uint32_t w = pos >> 5, b = pos & 31;
  uint64_t v = 0;
  if (w < 8) v = s[w];
  if (w + 1 < 8) v |= (uint64_t)s[w + 1] << 32;
  return (uint32_t)(v >> b) & ((1u << c) - 1u);
}

// Signed digits of one scalar, low window first; calls f(w, digit) for
// each non-zero digit (digit in [-2^(c-1), 2^(c-1)]).
template <class F>
__device__ __forceinline__ void for_each_digit(const fe* scalar, uint32_t c, uint32_t windows, F f) {
  uint32_t s[8];
  ld_fe(s, scalar);
  uint32_t one[8] = {1, 0, 0, 0, 0, 0, 0, 0};
  mul<FrP>(s, s, one);  // out of Montgomery form (cuda/curve.cuh:111 does the same)
  const int half = 1 << (c - 1);
  uint32_t carry = 0;
  for (uint32_t w = 0; w < windows; w++) {
    int v = (int)scalar_bits(s, w * c, c) + (int)carry;
    if (v > half) {
      v -= 1 << c;
      carry = 1;
    } else {
      carry = 0;
    }
    if (v != 0) f(w, v);
  }
}

// Several MSMs over one base array in one pass: scalars of job j occupy
// [off[j], off[j+1]) of the concatenated scalar array, its windows are
// j * windows + w, and its entries name the base by the local index.
__device__ __forceinline__ uint32_t job_of(const uint32_t* off, uint32_t jobs, uint32_t i) {
  uint32_t lo = 0, hi = jobs;  // off[lo] <= i < off[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= i) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void msm_count_kernel(const fe* scalars, uint64_t n, uint32_t c, uint32_t windows, uint32_t* counts,
                                 const uint32_t* job_off, uint32_t jobs) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t B = 1u << (c - 1);
  const uint32_t w0 = jobs > 1 ? job_of(job_off, jobs, (uint32_t)i) * windows : 0u;
  for_each_digit(scalars + i, c, windows, [&](uint32_t w, int d) {
    const uint32_t mag = (uint32_t)(d < 0 ? -d : d);
    atomicAdd(&counts[(w0 + w) * B + mag - 1], 1u);
  });
}

__global__ void msm_scatter_kernel(const fe* scalars, uint64_t n, uint32_t c, uint32_t windows, uint32_t* cursor,
                                   uint32_t* list, const uint32_t* job_off, uint32_t jobs) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t B = 1u << (c - 1);
  uint32_t w0 = 0, local = (uint32_t)i;
  if (jobs > 1) {
    const uint32_t j = job_of(job_off, jobs, (uint32_t)i);
    w0 = j * windows;
    local = (uint32_t)i - job_off[j];
  }
  for_each_digit(scalars + i, c, windows, [&](uint32_t w, int d) {
    const uint32_t mag = (uint32_t)(d < 0 ? -d : d);
    const uint32_t pos = atomicAdd(&cursor[(w0 + w) * B + mag - 1], 1u);
    list[pos] = local | (d < 0 ? 0x80000000u : 0u);
  });
}

// Exclusive scan, three phases over 1024-element blocks.
__global__ void scan_block_kernel(const uint32_t* in, uint32_t* out, uint32_t* block_sums, uint32_t total) {
  __shared__ uint32_t sh[1024];
  const uint32_t i = blockIdx.x * 1024 + threadIdx.x;
  const uint32_t v = i < total ? in[i] : 0;
  sh[threadIdx.x] = v;
  __syncthreads();
  for (uint32_t off = 1; off < 1024; off <<= 1) {
    uint32_t t = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < total) out[i] = sh[threadIdx.x] - v;
  if (threadIdx.x == 1023) block_sums[blockIdx.x] = sh[1023];
}
__global__ void scan_sums_kernel(uint32_t* block_sums, uint32_t nblocks, uint32_t* total_out) {
  // one block of 1024 threads; nblocks <= 1024 * 64
  __shared__ uint32_t sh[1024];
  uint32_t carry = 0;
  for (uint32_t base = 0; base < nblocks; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < nblocks ? block_sums[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
      uint32_t t = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nblocks) block_sums[i] = carry + sh[threadIdx.x] - v;
    const uint32_t tot = sh[1023];
    __syncthreads();
    carry += tot;
  }
  if (threadIdx.x == 0) *total_out = carry;
}
__global__ void scan_add_kernel(uint32_t* out, uint32_t* cursor, const uint32_t* block_sums, uint32_t total) {
  const uint32_t i = blockIdx.x * 1024 + threadIdx.x;
  if (i >= total) return;
  const uint32_t v = out[i] + block_sums[blockIdx.x];
  out[i] = v;
  cursor[i] = v;
}

// ---------------------------------------------------------------------------
// Batch-affine bucket accumulation.
//
// Every bucket's points are summed by pairwise AFFINE additions in rounds:
// round r replaces the c points of a bucket by ceil(c / 2) points (pair sums,
// plus the odd last point carried).  An affine addition P + Q needs
// 1 / (x_Q - x_P); the inverses of a whole round come from Montgomery's
// trick in two levels:
//   prefix  : each thread task owns BA_K consecutive pair sums and chains
//             the products of their denominators (stored, 1 product each);
//   invert  : each inversion thread takes BA_G task products, chains them,
//             inverts the chain's product once (Fermat) and walks back;
//   apply   : each task walks its chain back (2 products per sum) and
//             finishes the additions (lambda, lambda^2, lambda (x1 - x3):
//             3 products).
// That is about 6 + 3 / BA_K ~ 6.2 Fq products per point addition (the XYZZ
// mixed addition costs 10) plus one inversion per 512 additions, done by
// the branch-free divstep algorithm of fq_inv.cuh (~25k instructions of
// 32-bit integer work against ~330 dependent products for a Fermat power),
// with no serial block-wide step.  Equal x
// (P = Q: doubling, denominator 2y; P = -Q: identity) and the identity
// (x = 0: no BN254 point has x = 0, as 3 is not a square mod q) are handled
// per sum.  A bucket reaching one point writes it to `fin`; after the last
// round a tail kernel folds what remains (skewed buckets) with XYZZ mixed
// additions and writes every bucket as XYZZ for the reduction.
// ---------------------------------------------------------------------------
constexpr uint32_t BA_K = 16;  // pair sums per task (one chain of products)
constexpr uint32_t BA_G = 32;  // task products per inversion

__device__ __forceinline__ void fq_one_rp(uint32_t r[8]) { set_one_rp<FqP>(r); }

// a^-1 for a != 0 in R' form (x 2^260), lazy in, canonical out: the divstep
// inversion (fq_inv.cuh) of the representative a 2^260 gives a^-1 2^-260,
// and one product with 2^780 mod q returns it to R' form.
__device__ __forceinline__ void fq_inv_rp_bin(uint32_t r[8], const uint32_t a[8]) {
  const uint32_t k780[8] = {0x3fe3a1a8u, 0x13e32478u, 0x6ad256c5u, 0xc59c2897u,
                            0x3603f972u, 0xc5387239u, 0x8d1987f5u, 0x10f16dedu};
  uint32_t c[8], t[8];
  reduce_once<FqP>(c, a);
  fq_inv_divsteps(t, c);
  qmul(r, t, k780);
  reduce_once<FqP>(r, r);
}

// ---- per-thread copy pipeline ---------------------------------------------
// The prefix and apply passes are chains of dependent gathers (bucket
// metadata -> entry list -> point) and field products.  Each thread stages
// the operands of its next pair sum into shared memory with cp.async (16-B
// copies that hold no registers while in flight) while it computes the
// current one, and loads the entry-list words one job further ahead, so the
// gather latency overlaps the products.  Stage slots are chunk-major: chunk
// k of stage s of thread t is the 16-B word ((s * CH + k) * blockDim + t),
// so the 16-B accesses of a warp to one chunk are 32 consecutive words.
// .cg: through L2 only; staged data is read once, so allocating it in L1
// only evicts other lines.  (Round 0's random 32-B and 64-B gathers move
// whole 128-B lines from DRAM either way: 6.5 GB of DRAM reads for 2.2 GB
// of x coordinates in the 2^22-point prefix pass, measured on B200.)
__device__ __forceinline__ void cp16(uint4* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// one fe (two chunks) of a stage: copy in, read out
__device__ __forceinline__ void cp_fe(uint4* my, uint32_t bd, uint32_t k, const fe* g) {
  const uint4* v = reinterpret_cast<const uint4*>(g);
  cp16(my + k * bd, v);
  cp16(my + (k + 1) * bd, v + 1);
}
__device__ __forceinline__ void sm_fe(uint32_t r[8], const uint4* my, uint32_t bd, uint32_t k) {
  const uint4 x = my[k * bd], y = my[(k + 1) * bd];
  r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
  r[4] = y.x; r[5] = y.y; r[6] = y.z; r[7] = y.w;
}

// one pair sum of a round: its two points in the round's source (round 0:
// entry-list words, base index plus sign bit; later rounds: positions in the
// previous round's output), its bucket, and whether the second point exists
constexpr uint32_t BA_CP = 4;   // chunks per prefix stage: x of both points
constexpr uint32_t BA_CA = 10;  // chunks per apply stage: both points, one prefix product
struct BaJob {
  uint32_t pa, pb, b;
  bool has2;
};

template <bool FIRST>
__device__ __forceinline__ BaJob ba_job(uint32_t q, uint32_t b, const uint32_t* __restrict__ joff,
                                        const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ cprev,
                                        const uint32_t* __restrict__ list) {
  BaJob d;
  const uint32_t j = q - joff[b];
  const uint32_t i0 = in_off[b] + 2 * j;
  d.b = b;
  d.has2 = 2 * j + 1 < cprev[b];
  if (FIRST) {
    d.pa = list[i0];
    d.pb = d.has2 ? list[i0 + 1] : 0u;
  } else {
    d.pa = i0;
    d.pb = i0 + 1;
  }
  return d;
}
// point p of a round's source ((x, y) adjacent): round 0 reads the bases
// (the entry's index, sign bit cleared), later rounds their own buffer of
// affine pair sums.  (Bases kept as an x array and a y array instead were
// measured on B200 at 2^22 points: the prefix pass's x gathers hit L2 more,
// 1.28 -> 1.15 ms, and the apply pass's separate y gathers cost as much,
// 3.94 -> 4.06 ms.)
template <bool FIRST>
__device__ __forceinline__ const fe* ba_pt(const fe* src, uint32_t p) {
  return src + 2 * (uint64_t)(FIRST ? (p & 0x7fffffffu) : p);
}
// y of a round-0 point read out of its slot: negated for a negative digit
template <bool FIRST>
__device__ __forceinline__ void ba_sign(aff_t& p, uint32_t e) {
  if (FIRST && (e & 0x80000000u) && !is_zero(p.x)) {
    uint32_t z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    sub<FqP>(p.y, z, p.y);
  }
}

// bucket of job q: the largest b' with joff[b'] <= q, searched from the
// bucket of a neighbouring job (forward: joff[b] <= q; backward: q < joff[b + 1])
__device__ __forceinline__ uint32_t ba_search(const uint32_t* __restrict__ joff, uint32_t lo, uint32_t hi,
                                              uint32_t q) {
  while (hi - lo > 1) {  // joff[lo] <= q < joff[hi]
    const uint32_t mid = (lo + hi) >> 1;
    if (joff[mid] <= q) lo = mid; else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ uint32_t ba_bucket_fwd(const uint32_t* __restrict__ joff, uint32_t T, uint32_t b,
                                                  uint32_t q) {
  if (joff[b + 1] > q) return b;
  if (b + 2 <= T && joff[b + 2] > q) return b + 1;
  return ba_search(joff, b + 1, T, q);
}
__device__ __forceinline__ uint32_t ba_bucket_bwd(const uint32_t* __restrict__ joff, uint32_t b, uint32_t q) {
  if (joff[b] <= q) return b;
  if (joff[b - 1] <= q) return b - 1;
  return ba_search(joff, 0, b - 1, q);
}

// stage the x coordinates of a job's points (prefix pass)
template <bool FIRST>
__device__ __forceinline__ void ba_stage_x(uint4* st, uint32_t bd, const fe* src, const BaJob& d) {
  if (!d.has2) return;
  cp_fe(st, bd, 0, ba_pt<FIRST>(src, d.pa));
  cp_fe(st, bd, 2, ba_pt<FIRST>(src, d.pb));
}
// stage both points of a job and the prefix product before it (apply pass)
template <bool FIRST>
__device__ __forceinline__ void ba_stage_pq(uint4* st, uint32_t bd, const fe* src, const BaJob& d, const fe* p) {
  const fe* a = ba_pt<FIRST>(src, d.pa);
  cp_fe(st, bd, 0, a);
  cp_fe(st, bd, 2, a + 1);
  if (d.has2) {
    const fe* c = ba_pt<FIRST>(src, d.pb);
    cp_fe(st, bd, 4, c);
    cp_fe(st, bd, 6, c + 1);
  }
  if (p) cp_fe(st, bd, 8, p);
}

// denominator of one pair sum (R' one when no inversion is needed: a carried
// point, an identity operand, or P = -Q), from the staged x coordinates;
// equal x (doubling or P = -Q, rare) reads both points again for y
template <bool FIRST>
__device__ __forceinline__ void ba_denominator(uint32_t d[8], const uint4* st, uint32_t bd, const fe* src,
                                               const BaJob& job) {
  if (job.has2) {
    uint32_t x1[8], x2[8];
    sm_fe(x1, st, bd, 0);
    sm_fe(x2, st, bd, 2);
    if (!is_zero(x1) && !is_zero(x2)) {
      if (!eq(x1, x2)) {
        sub<FqP>(d, x2, x1);
        return;
      }
      aff_t p, q;
      ld_aff(p, ba_pt<FIRST>(src, job.pa));
      ld_aff(q, ba_pt<FIRST>(src, job.pb));
      ba_sign<FIRST>(p, job.pa);
      ba_sign<FIRST>(q, job.pb);
      if (eq(p.y, q.y)) {
        add<FqP>(d, p.y, p.y);
        return;
      }
    }
  }
  fq_one_rp(d);
}

// buckets with at most one entry are final before any round; every count
// is copied for the rounds
__global__ void ba_setup_kernel(const uint32_t* counts, const uint32_t* offsets, const uint32_t* list,
                                const fe* bases, uint32_t* cnt, fe* fin, uint32_t T) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= T) return;
  const uint32_t c = counts[b];
  cnt[b] = c;
  if (c == 1) {
    aff_t p;
    const uint32_t e = list[offsets[b]];
    ld_aff(p, ba_pt<true>(bases, e));
    ba_sign<true>(p, e);
    st_fe(fin + 2 * (uint64_t)b, p.x);
    st_fe(fin + 2 * (uint64_t)b + 1, p.y);
  } else if (c == 0) {
    uint32_t z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    st_fe(fin + 2 * (uint64_t)b, z);
    st_fe(fin + 2 * (uint64_t)b + 1, z);
  }
}

__global__ void ba_jobs_kernel(const uint32_t* cnt, uint32_t* cprev, uint32_t* np, uint32_t T) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= T) return;
  const uint32_t c = cnt[b];
  cprev[b] = c;
  np[b] = c >= 2 ? (c + 1) / 2 : 0;
}

// prefix: task t covers jobs [t K, t K + K) of the round (J = joff[T])
// pair sums per task in a round of J sums: BA_K when the round fills the GPU
// with tasks, fewer (down to one) in small rounds, whose latency is then one
// short chain instead of BA_K dependent gathers and products
__device__ __forceinline__ uint32_t ba_task_len(uint32_t J, uint32_t fill_k) {
  return max(1u, min(BA_K, J / fill_k));
}

// dynamic shared memory: 2 stages x BA_CP chunks x 16 B per thread
template <bool FIRST>
__global__ void __launch_bounds__(256) ba_prefix_kernel(const fe* __restrict__ src, const uint32_t* __restrict__ list,
                                                        const uint32_t* __restrict__ in_off,
                                                        const uint32_t* __restrict__ cprev,
                                                        const uint32_t* __restrict__ joff, uint32_t T,
                                                        fe* __restrict__ pre, fe* __restrict__ tot,
                                                        uint32_t fill_k) {
  extern __shared__ uint4 ba_smem[];
  const uint32_t bd = blockDim.x;
  uint4* my = ba_smem + threadIdx.x;
  const uint32_t J = joff[T];
  const uint32_t K = ba_task_len(J, fill_k);
  const uint32_t tasks = (J + K - 1) / K;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < tasks; t += gridDim.x * blockDim.x) {
    const uint32_t q0 = t * K, q1 = min(q0 + K, J);
    uint32_t b = ba_search(joff, 0, T, q0);
    BaJob d0 = ba_job<FIRST>(q0, b, joff, in_off, cprev, list), d1 = d0;
    ba_stage_x<FIRST>(my, bd, src, d0);
    cp_commit();
    if (q0 + 1 < q1) {
      b = ba_bucket_fwd(joff, T, b, q0 + 1);
      d1 = ba_job<FIRST>(q0 + 1, b, joff, in_off, cprev, list);
    }
    uint32_t acc[8];
    for (uint32_t q = q0; q < q1; q++) {
      const uint32_t s = (q - q0) & 1;
      if (q + 1 < q1) ba_stage_x<FIRST>(my + (s ^ 1) * BA_CP * bd, bd, src, d1);
      cp_commit();
      BaJob d2 = d1;
      if (q + 2 < q1) {
        b = ba_bucket_fwd(joff, T, b, q + 2);
        d2 = ba_job<FIRST>(q + 2, b, joff, in_off, cprev, list);
      }
      cp_wait<1>();
      uint32_t d[8];
      ba_denominator<FIRST>(d, my + s * BA_CP * bd, bd, src, d0);
      if (q == q0)
        cpy(acc, d);
      else
        qmul(acc, acc, d);
      st_fe(pre + q, acc);
      d0 = d1;
      d1 = d2;
    }
    st_fe(tot + t, acc);
  }
  cp_wait<0>();
}

// invert: thread s turns tot[s G .. s G + G) into their inverses.  The
// group length G follows the round's size: up to BA_G task products per
// inversion when there are many, down to one when a round is small, so that
// the round's latency is one inversion plus a short chain.
__global__ void __launch_bounds__(128) ba_invert_kernel(fe* tot, fe* tpre, const uint32_t* joff, uint32_t T,
                                                        uint32_t fill, uint32_t fill_k) {
  const uint32_t J = joff[T];
  const uint32_t K = ba_task_len(J, fill_k);
  const uint32_t tasks = (J + K - 1) / K;
  const uint32_t G = max(1u, min(BA_G, tasks / fill));
  const uint32_t groups = (tasks + G - 1) / G;
  for (uint32_t sgi = blockIdx.x * blockDim.x + threadIdx.x; sgi < groups; sgi += gridDim.x * blockDim.x) {
    const uint32_t i0 = sgi * G, i1 = min(i0 + G, tasks);
    uint32_t acc[8], v[8];
    ld_fe(acc, tot + i0);
    st_fe(tpre + i0, acc);
    for (uint32_t i = i0 + 1; i < i1; i++) {
      ld_fe(v, tot + i);
      qmul(acc, acc, v);
      st_fe(tpre + i, acc);
    }
    uint32_t inv[8];
    fq_inv_rp_bin(inv, acc);
    for (uint32_t i = i1 - 1; i > i0; i--) {
      uint32_t p[8], it[8];
      ld_fe(p, tpre + i - 1);
      ld_fe(v, tot + i);
      qmul(it, inv, p);
      qmul(inv, inv, v);
      st_fe(tot + i, it);
    }
    st_fe(tot + i0, inv);
  }
}

// apply: walk each task's chain back and finish its pair sums; dynamic
// shared memory: 2 stages x BA_CA chunks x 16 B per thread
template <bool FIRST>
__global__ void __launch_bounds__(256, 2) ba_apply_kernel(const fe* __restrict__ src,
                                                          const uint32_t* __restrict__ list,
                                                          const uint32_t* __restrict__ in_off,
                                                          const uint32_t* __restrict__ cprev,
                                                          const uint32_t* __restrict__ joff,
                                                          const uint32_t* __restrict__ np, uint32_t T,
                                                          const fe* __restrict__ pre, const fe* __restrict__ tot,
                                                          fe* __restrict__ dst, fe* __restrict__ fin,
                                                          uint32_t* __restrict__ cnt, uint32_t fill_k) {
  extern __shared__ uint4 ba_smem[];
  const uint32_t bd = blockDim.x;
  uint4* my = ba_smem + threadIdx.x;
  const uint32_t J = joff[T];
  const uint32_t K = ba_task_len(J, fill_k);
  const uint32_t tasks = (J + K - 1) / K;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < tasks; t += gridDim.x * blockDim.x) {
    const uint32_t q0 = t * K, q1 = min(q0 + K, J);
    uint32_t inv_run[8];
    ld_fe(inv_run, tot + t);
    uint32_t b = ba_search(joff, 0, T, q1 - 1);
    BaJob d0 = ba_job<FIRST>(q1 - 1, b, joff, in_off, cprev, list), d1 = d0;
    ba_stage_pq<FIRST>(my, bd, src, d0, q1 - 1 > q0 ? pre + q1 - 2 : nullptr);
    cp_commit();
    if (q1 - 1 > q0) {
      b = ba_bucket_bwd(joff, b, q1 - 2);
      d1 = ba_job<FIRST>(q1 - 2, b, joff, in_off, cprev, list);
    }
    for (uint32_t q = q1, i = 0; q-- > q0; i++) {
      const uint32_t s = i & 1;
      if (q > q0) ba_stage_pq<FIRST>(my + (s ^ 1) * BA_CA * bd, bd, src, d1, q - 1 > q0 ? pre + q - 2 : nullptr);
      cp_commit();
      BaJob d2 = d1;
      if (q > q0 + 1) {
        b = ba_bucket_bwd(joff, b, q - 2);
        d2 = ba_job<FIRST>(q - 2, b, joff, in_off, cprev, list);
      }
      cp_wait<1>();
      const uint4* st = my + s * BA_CA * bd;
      const bool has2 = d0.has2;
      aff_t P, Q, out;
      sm_fe(P.x, st, bd, 0);
      sm_fe(P.y, st, bd, 2);
      ba_sign<FIRST>(P, d0.pa);
      if (has2) {
        sm_fe(Q.x, st, bd, 4);
        sm_fe(Q.y, st, bd, 6);
        ba_sign<FIRST>(Q, d0.pb);
      }
      // the same denominator the prefix pass chained (ba_denominator)
      uint32_t d[8];
      int kind = 0;  // 0: no inversion, 1: addition, 2: doubling
      if (has2 && !is_zero(P.x) && !is_zero(Q.x)) {
        if (!eq(P.x, Q.x)) {
          sub<FqP>(d, Q.x, P.x);
          kind = 1;
        } else if (eq(P.y, Q.y)) {
          add<FqP>(d, P.y, P.y);
          kind = 2;
        }
      }
      if (kind == 0) fq_one_rp(d);
      uint32_t inv_d[8];
      if (q > q0) {
        uint32_t p[8];
        sm_fe(p, st, bd, 8);
        qmul_c(inv_d, inv_run, p);
        qmul_c(inv_run, inv_run, d);
      } else {
        cpy(inv_d, inv_run);
      }
      if (!has2 || is_zero(Q.x)) {
        out = P;
      } else if (is_zero(P.x)) {
        out = Q;
      } else if (kind == 0) {  // P = -Q
        set_zero(out.x);
        set_zero(out.y);
      } else {
        uint32_t lam[8], t1[8];
        if (kind == 1) {
          sub<FqP>(t1, Q.y, P.y);
        } else {  // doubling: 3 x^2 / (2 y)
          qsqr_c(t1, P.x);
          uint32_t t2[8];
          add_lazy<FqP>(t2, t1, t1);
          add_lazy<FqP>(t1, t2, t1);
        }
        qmul_c(lam, t1, inv_d);
        qsqr_c(t1, lam);
        qsub(t1, t1, P.x);
        qsub(out.x, t1, Q.x);  // Q.x = P.x when doubling
        reduce_once<FqP>(out.x, out.x);
        qsub(t1, P.x, out.x);
        qmul_c(t1, lam, t1);
        qsub(out.y, t1, P.y);
        reduce_once<FqP>(out.y, out.y);
      }
      const uint32_t bq = d0.b, nb = np[bq];
      fe* o = nb == 1 ? fin + 2 * (uint64_t)bq : dst + 2 * (uint64_t)q;
      st_fe(o, out.x);
      st_fe(o + 1, out.y);
      if (q == joff[bq]) cnt[bq] = nb;
      d0 = d1;
      d1 = d2;
    }
  }
  cp_wait<0>();
}

// Tail: what the rounds left (a few points per bucket, or many in a skewed
// bucket such as the one small scalars carry into) is folded with XYZZ mixed
// additions in chunks of BA_TS points, one thread per chunk; a bucket's
// chunk sums are then added by one thread, or block-wide when there are many.
constexpr uint32_t BA_TS = 16;    // points per tail chunk
constexpr uint32_t BA_TSEQ = 16;  // chunk sums a bucket adds in one thread

__global__ void ba_chunks_kernel(const uint32_t* cnt, uint32_t* nch, uint32_t T) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= T) return;
  const uint32_t c = cnt[b];
  nch[b] = c <= 1 ? 1u : (c + BA_TS - 1) / BA_TS;
}

__global__ void __launch_bounds__(256) ba_fold_kernel(const uint32_t* cnt, const uint32_t* in_off, const fe* src,
                                                      const fe* fin, const uint32_t* coff, const uint32_t* nch,
                                                      uint32_t T, fe* chunk_res) {
  const uint32_t C = coff[T];
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < C; u += gridDim.x * blockDim.x) {
    const uint32_t b = ba_search(coff, 0, T, u);
    const uint32_t k = u - coff[b], c = cnt[b];
    xyzz_t acc;
    xyzz_set_inf(acc);
    aff_t p;
    if (c <= 1) {
      ld_aff(p, fin + 2 * (uint64_t)b);
      xyzz_from_aff(acc, p);  // (0, 0) -> identity
    } else {
      const uint32_t o = in_off[b], i1 = min(c, (k + 1) * BA_TS);
      for (uint32_t i = k * BA_TS; i < i1; i++) {
        ld_aff(p, src + 2 * (uint64_t)(o + i));
        xyzz_madd(acc, p);
      }
    }
    st_xyzz(chunk_res + 4 * (uint64_t)u, acc);
  }
}

__global__ void ba_bucket_sum_kernel(const uint32_t* coff, const uint32_t* nch, const fe* chunk_res, fe* buckets,
                                     uint32_t* heavy, uint32_t* heavy_count, uint32_t T) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= T) return;
  const uint32_t k = nch[b], o = coff[b];
  if (k > BA_TSEQ) {
    heavy[atomicAdd(heavy_count, 1u)] = b;
    return;
  }
  xyzz_t acc, t;
  ld_xyzz(acc, chunk_res + 4 * (uint64_t)o);
  for (uint32_t j = 1; j < k; j++) {
    ld_xyzz(t, chunk_res + 4 * (uint64_t)(o + j));
    xyzz_add(acc, t);
  }
  st_xyzz(buckets + 4 * (uint64_t)b, acc);
}

// One block per queued heavy bucket: strided partial sums, then a tree.
__global__ void __launch_bounds__(256) ba_heavy_kernel(const uint32_t* coff, const uint32_t* nch, const fe* chunk_res,
                                                       fe* buckets, const uint32_t* heavy,
                                                       const uint32_t* heavy_count) {
  __shared__ fe sh[256 * 4];
  if (blockIdx.x >= *heavy_count) return;
  const uint32_t b = heavy[blockIdx.x];
  const uint32_t k = nch[b], o = coff[b];
  xyzz_t acc, t;
  xyzz_set_inf(acc);
  for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
    ld_xyzz(t, chunk_res + 4 * (uint64_t)(o + j));
    xyzz_add(acc, t);
  }
  st_xyzz(sh + 4 * threadIdx.x, acc);
  __syncthreads();
  for (uint32_t half = blockDim.x / 2; half > 0; half >>= 1) {
    if (threadIdx.x < half) {
      ld_xyzz(acc, sh + 4 * threadIdx.x);
      ld_xyzz(t, sh + 4 * (threadIdx.x + half));
      xyzz_add(acc, t);
      st_xyzz(sh + 4 * threadIdx.x, acc);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ld_xyzz(acc, sh);
    st_xyzz(buckets + 4 * (uint64_t)b, acc);
  }
}

// Bucket reduction.  A window's sum is W = sum_j (j + 1) B_j over its B
// buckets.  Level 1, one thread per segment of L buckets: running sums from
// the top give T_s = sum_i (i + 1) B_{sL+i} and S_s = sum_i B_{sL+i}, so
// W = sum_s T_s + L sum_s s S_s.
__global__ void __launch_bounds__(128) msm_segment_kernel(const fe* buckets, fe* seg_t, fe* seg_s, uint32_t B,
                                                          uint32_t L, uint32_t total_segs) {
  const uint32_t gs = blockIdx.x * blockDim.x + threadIdx.x;
  if (gs >= total_segs) return;
  const uint32_t S_per_w = B / L;
  const uint32_t w = gs / S_per_w, s = gs % S_per_w;
  const uint32_t lo = s * L;
  xyzz_t run, tot, bk;
  xyzz_set_inf(run);
  xyzz_set_inf(tot);
  for (int j = (int)(lo + L) - 1; j >= (int)lo; j--) {
    ld_xyzz(bk, buckets + 4 * ((uint64_t)w * B + j));
    xyzz_add(run, bk);
    xyzz_add(tot, run);
  }
  st_xyzz(seg_t + 4 * (uint64_t)gs, tot);
  st_xyzz(seg_s + 4 * (uint64_t)gs, run);
}

// Level 2, one block per window, thread t owning M consecutive segments
// (S_per_w and the block size are powers of two): A_t = sum_k T_{tM+k},
// U_t = sum_k k S_{tM+k} and V_t = sum_k S_{tM+k} by running sums, so that
// sum_s s S_s = sum_t U_t + M sum_t t V_t, and sum_t t V_t = sum_{t>=1} P_t
// with P_t = sum_{u>=t} V_u (a block suffix scan).  Thread t contributes
// c_t = A_t + L U_t + L M P_t (no P term for t = 0); a tree sum gives W.
// The serial depth is about M + 2 log2(256) additions and log2(L M)
// doublings per window, against L + c doublings and additions per segment
// for multiplying every segment sum by its offset (measured on B200, 2^22
// points, c = 16: 1.16 ms for both levels against 1.25 ms).  The
// accumulator not being added to waits in the thread's slot of shared
// memory (two slot arrays, 64 KiB of dynamic shared memory), so at most
// two points are live in registers.
constexpr int kWindowSmem = 2 * 256 * 128;
__global__ void __launch_bounds__(256) msm_window_kernel(const fe* seg_t, const fe* seg_s, fe* winsum,
                                                         uint32_t S_per_w, uint32_t L) {
  extern __shared__ uint4 win_smem[];
  fe* sc = reinterpret_cast<fe*>(win_smem);  // per thread: c_t, then the tree
  fe* sv = sc + 4 * blockDim.x;               // per thread: V_t, then the scan
  const uint32_t w = blockIdx.x, t = threadIdx.x, nt = blockDim.x;
  const uint32_t M = S_per_w > nt ? S_per_w / nt : 1u;
  const uint32_t active = S_per_w / M;
  xyzz_t a, x;
  xyzz_set_inf(a);
  st_xyzz(sc + 4 * t, a);  // U_t accumulates here
  if (t < active) {
    const uint64_t base = (uint64_t)w * S_per_w + (uint64_t)t * M;
    // a = V (running), U in sc
    for (uint32_t k = M - 1; k >= 1; k--) {
      ld_xyzz(x, seg_s + 4 * (base + k));
      xyzz_add(a, x);
      ld_xyzz(x, sc + 4 * t);
      xyzz_add(x, a);
      st_xyzz(sc + 4 * t, x);
    }
    ld_xyzz(x, seg_s + 4 * base);
    xyzz_add(a, x);
    st_xyzz(sv + 4 * t, a);  // V_t
    // a = L U_t + A_t
    ld_xyzz(a, sc + 4 * t);
    for (uint32_t m = L; m > 1; m >>= 1) xyzz_dbl(a, a);  // L a power of two
    for (uint32_t k = 0; k < M; k++) {
      ld_xyzz(x, seg_t + 4 * (base + k));
      xyzz_add(a, x);
    }
  } else {
    st_xyzz(sv + 4 * t, a);
  }
  st_xyzz(sc + 4 * t, a);
  __syncthreads();
  // suffix sums of V across the block
  ld_xyzz(a, sv + 4 * t);
  for (uint32_t off = 1; off < nt; off <<= 1) {
    const bool has = t + off < nt;
    if (has) ld_xyzz(x, sv + 4 * (t + off));
    __syncthreads();
    if (has) {
      xyzz_add(a, x);
      st_xyzz(sv + 4 * t, a);
    }
    __syncthreads();
  }
  if (t > 0) {
    for (uint32_t m = L * M; m > 1; m >>= 1) xyzz_dbl(a, a);  // L M P_t
    ld_xyzz(x, sc + 4 * t);
    xyzz_add(x, a);
    st_xyzz(sc + 4 * t, x);
  }
  __syncthreads();
  for (uint32_t half = nt / 2; half > 0; half >>= 1) {
    if (t < half) {
      ld_xyzz(a, sc + 4 * t);
      ld_xyzz(x, sc + 4 * (t + half));
      xyzz_add(a, x);
      st_xyzz(sc + 4 * t, a);
    }
    __syncthreads();
  }
  if (t == 0) {
    ld_xyzz(a, sc);
    st_xyzz(winsum + 4 * (uint64_t)w, a);
  }
}

// bases (R form, as the API holds them) -> R' form for the curve arithmetic
__global__ void msm_convert_bases_kernel(const fe* in, fe* out, uint64_t n) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t x[8], y[8];
  ld_fe(x, in + 2 * i);
  ld_fe(y, in + 2 * i + 1);
  to_rprime(x, x);
  to_rprime(y, y);
  st_fe(out + 2 * i, x);
  st_fe(out + 2 * i + 1, y);
}

__global__ void zero_out_kernel(fe* out) {
  if (threadIdx.x < 3) {
    uint32_t z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    st_fe(out + threadIdx.x, z);
  }
}

namespace {
// The Horner step over the window sums (sum_w 2^(c w) W_w, ~250 dependent
// doublings) is serial: one GPU thread needs over a millisecond for it, the
// host well under 0.1 ms.  The device-resident call keeps stream order and
// asynchrony by running it as a host function on the stream: window sums to
// a pinned slot, host_horner() on the stream, the normalised Jacobian result
// back to the caller's device buffer.  Slots are per host thread and reused
// round robin once the event of their last use has completed.
struct HornerSlot {
  uint64_t win[MSM_MAX_WINDOWS * 16];
  uint64_t out[12];
  uint32_t windows = 0, c = 0;
  cudaEvent_t done = nullptr;
};
constexpr int kHornerSlots = 8;
struct HornerRing {
  HornerSlot* slots = nullptr;  // pinned, kHornerSlots entries
  int next = 0;
};
thread_local HornerRing t_horner;

void CUDART_CB host_horner(void* arg) {
  HornerSlot* h = static_cast<HornerSlot*>(arg);
  host::fq::msm_combine_windows(h->win, h->windows, h->c, h->out);
}

cudaError_t horner_on_host(const fe* d_winsum, uint32_t windows, uint32_t c, fe* d_out, cudaStream_t s) {
  HornerRing& r = t_horner;
  if (!r.slots) {
    cudaError_t e = cudaMallocHost((void**)&r.slots, sizeof(HornerSlot) * kHornerSlots);
    if (e != cudaSuccess) return e;
    for (int i = 0; i < kHornerSlots; i++) {
      new (&r.slots[i]) HornerSlot();
      e = cudaEventCreateWithFlags(&r.slots[i].done, cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
  }
  HornerSlot* h = &r.slots[r.next];
  r.next = (r.next + 1) % kHornerSlots;
  cudaError_t e = cudaEventSynchronize(h->done);  // its last use has finished (normally long ago)
  if (e != cudaSuccess) return e;
  h->windows = windows;
  h->c = c;
  e = cudaMemcpyAsync(h->win, d_winsum, windows * 128ull, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaLaunchHostFunc(s, host_horner, h);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, h->out, 96, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaEventRecord(h->done, s);
  return e;
}

// tasks of a round of at most jb pair sums (ba_task_len: K = clamp(J / fill_k, 1, BA_K))
uint64_t ba_tasks_bound(uint64_t jb, uint64_t fill_k) {
  return std::max<uint64_t>(2 * fill_k, jb / BA_K + 1);
}
constexpr uint32_t kFillK = 148 * 64;  // task threads that fill a B200 (148 SMs) at 64 per SM

// dynamic shared memory of the round kernels at 256 threads (two stages)
constexpr int kPrefixSmem = 2 * BA_CP * 16 * 256;  // 32 KiB
constexpr int kApplySmem = 2 * BA_CA * 16 * 256;   // 80 KiB: above the 48 KiB default, opted in per device
// (as is the window kernel's kWindowSmem, 64 KiB)

cudaError_t ba_kernel_attrs(int device) {
  static std::mutex mu;
  static uint64_t done = 0;  // one bit per device
  std::lock_guard<std::mutex> lk(mu);
  if (device < 64 && (done >> device) & 1) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(ba_apply_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kApplySmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ba_apply_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kApplySmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(msm_window_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kWindowSmem);
  if (e == cudaSuccess && device < 64) done |= 1ull << device;
  return e;
}

// Buffer sizes of one MSM pass (msm_run_impl allocates exactly these;
// msm_scratch_bytes reports them for admission).
struct MsmLayout {
  MsmPlan p;
  uint32_t Wj = 0, W = 0, B = 0, L = 0, T = 0, nblk = 0, segs = 0, rounds = 0;
  uint64_t E = 0;                // entries (point-window pairs), upper bound
  uint64_t jb[2] = {0, 0};       // pair sums of rounds 0 and 1, upper bounds
  uint64_t tasks0 = 0;
  uint64_t chunks = 0;           // tail chunks, upper bound
  bool ok = false;
  uint64_t bytes(bool own_winsum, uint64_t nbases_convert) const {
    const uint64_t T1 = T + 1ull;
    uint64_t b = 0;
    b += T * 4ull * 2 + T1 * 4 + (nblk + 1ull) * 4 + E * 4;        // counts, cursor, offsets, bsums, list
    b += T * 4ull * 3 + T1 * 4 * 2 + T * 64ull;                   // cnt, cprev, np, joff x2, fin
    b += jb[0] * 64 + (rounds > 1 ? jb[1] * 64 : 0) + jb[0] * 32;  // round buffers, prefixes
    b += tasks0 * 32 * 2;                                         // task products, their prefixes
    b += T * 4ull * 2 + chunks * 128 + 4;                         // tail: chunk counts, heavy list, chunk sums
    b += T * 128ull + segs * 256ull + (own_winsum ? W * 128ull : 0);  // buckets, segment T_s and S_s
    b += nbases_convert * 64;
    return b + 24 * 256;  // pool granularity per allocation
  }
};

MsmLayout msm_layout(uint64_t n, uint32_t jobs, int c_override, int device = -1) {
  MsmLayout l;
  if (jobs == 0) jobs = 1;
  l.p = make_msm_plan((n + jobs - 1) / jobs, c_override, device);  // one window size: the mean job size's plan
  l.Wj = (uint32_t)l.p.windows;
  l.B = l.p.buckets;
  l.L = l.p.seg_len;
  const uint64_t W = (uint64_t)l.Wj * jobs;
  if (W * l.B >= (1ull << 31)) return l;
  l.W = (uint32_t)W;
  l.T = l.W * l.B;
  l.nblk = (l.T + 1023) / 1024;
  if (l.nblk > 1024u * 64u) return l;  // the three-phase scan's limit
  l.segs = l.T / l.L;
  l.E = n * (uint64_t)l.Wj;
  if (l.E >= (1ull << 32)) return l;  // entry offsets are 32-bit; pair sums < E / 2 + T < 2^32
  // rounds: enough to bring a bucket of the mean size plus a wide margin to
  // one point; anything left after them is folded by the tail kernel
  const uint64_t mean = (l.E + l.T - 1) / l.T;
  uint32_t lg = 0;
  while ((1ull << lg) < mean) lg++;
  // batch-affine rounds while buckets hold more than about four points;
  // later levels cost more in per-round latency than they save
  l.rounds = lg > 3 ? lg - 2 : 1;
  l.jb[0] = l.E / 2 + l.T;
  l.jb[1] = l.jb[0] / 2 + l.T;
  l.tasks0 = ba_tasks_bound(l.jb[0], kFillK);
  uint64_t jlast = l.jb[0];
  for (uint32_t r = 1; r < l.rounds; r++) jlast = jlast / 2 + l.T;
  l.chunks = l.T + jlast / BA_TS + 1;  // bound on sum_b max(1, ceil(cnt_b / BA_TS))
  l.ok = true;
  return l;
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// n: scalars (all jobs); jobs > 1: job_off (device, jobs + 1 entries) splits
// them and every job reads bases [0, nbases); the window sums of job j are
// windows [j W, (j + 1) W) of wout.  bases_rp_given: the bases are already in
// the R' form of the curve arithmetic (resident bases converted once).
cudaError_t msm_run_impl(const fe* d_scalars, const fe* d_bases, uint64_t n, fe* d_out, cudaStream_t s,
                         int c_override, uint64_t* launches, MsmWindowsOut* wout, const uint32_t* job_off,
                         uint32_t jobs, uint64_t nbases, bool bases_rp_given) {
  uint64_t nl = 0;
  if (n == 0) {
    if (wout) {
      wout->windows = 0;
      if (launches) *launches = 0;
      return cudaSuccess;
    }
    zero_out_kernel<<<1, 32, 0, s>>>(d_out);
    if (launches) *launches = 1;
    return cudaGetLastError();
  }
  if (jobs == 0) jobs = 1;
  const MsmLayout l = msm_layout(n, jobs, c_override);
  if (!l.ok) return cudaErrorInvalidValue;
  const MsmPlan& p = l.p;
  if (wout) {
    if ((uint32_t)p.windows > MSM_MAX_WINDOWS || !wout->d_winsum) return cudaErrorInvalidValue;
    wout->windows = (uint32_t)p.windows;
    wout->c = (uint32_t)p.c;
  }
  const uint32_t Wj = l.Wj, B = l.B, L = l.L, W = l.W, T = l.T, nblk = l.nblk, segs = l.segs;
  const uint64_t entries = l.E;
  uint32_t *counts = nullptr, *offsets = nullptr, *cursor = nullptr, *bsums = nullptr, *list = nullptr;
  uint32_t *cnt = nullptr, *cprev = nullptr, *np = nullptr, *joff[2] = {nullptr, nullptr};
  fe *fin = nullptr, *buf[2] = {nullptr, nullptr}, *pre = nullptr, *tot = nullptr, *tpre = nullptr;
  fe *buckets = nullptr, *segres = nullptr, *segsum = nullptr, *winsum = nullptr, *bases_rp = nullptr;
  fe* chunk_res = nullptr;
  uint32_t *nch = nullptr, *heavy = nullptr, *heavy_count = nullptr;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** ptr, size_t bytes) {
    if (e == cudaSuccess) e = zk::dmalloc(ptr, bytes ? bytes : 4, s);
  };
  alloc((void**)&counts, T * 4ull);
  alloc((void**)&offsets, (T + 1ull) * 4);
  alloc((void**)&cursor, T * 4ull);
  alloc((void**)&bsums, (nblk + 1ull) * 4);
  alloc((void**)&list, entries * 4ull);
  alloc((void**)&cnt, T * 4ull);
  alloc((void**)&cprev, T * 4ull);
  alloc((void**)&np, T * 4ull);
  alloc((void**)&joff[0], (T + 1ull) * 4);
  alloc((void**)&joff[1], (T + 1ull) * 4);
  alloc((void**)&fin, T * 64ull);
  alloc((void**)&buf[0], l.jb[0] * 64);
  if (l.rounds > 1) alloc((void**)&buf[1], l.jb[1] * 64);
  alloc((void**)&pre, l.jb[0] * 32);
  alloc((void**)&tot, l.tasks0 * 32);
  alloc((void**)&tpre, l.tasks0 * 32);
  alloc((void**)&nch, T * 4ull);
  alloc((void**)&heavy, T * 4ull);
  alloc((void**)&heavy_count, 4);
  alloc((void**)&chunk_res, l.chunks * 128);
  alloc((void**)&buckets, T * 128ull);
  alloc((void**)&segres, segs * 128ull);
  alloc((void**)&segsum, segs * 128ull);
  if (wout)
    winsum = wout->d_winsum;  // caller's buffer, left for the host's Horner step
  else
    alloc((void**)&winsum, W * 128ull);
  if (!bases_rp_given) alloc((void**)&bases_rp, nbases * 64ull);
  if (e == cudaSuccess) {
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = ba_kernel_attrs(dev);
  }
  if (e == cudaSuccess) {
    const double nd = (double)n;
    const int sms = sm_count();
    const uint32_t fill_k = kFillK;  // matches the task buffers' bound (layout)
    cudaMemsetAsync(counts, 0, T * 4ull, s);
    const unsigned g = (unsigned)((n + 255) / 256);
    const unsigned gb = (T + 255) / 256;
    const fe* bases = d_bases;
    if (!bases_rp_given) {
      msm_convert_bases_kernel<<<(unsigned)((nbases + 255) / 256), 256, 0, s>>>(d_bases, bases_rp, nbases);
      bases = bases_rp;
      nl++;
    }
    {
      ProfScope ps("msm_count", s, nd, nd * 32);
      msm_count_kernel<<<g, 256, 0, s>>>(d_scalars, n, (uint32_t)p.c, Wj, counts, job_off, jobs);
    }
    scan_block_kernel<<<nblk, 1024, 0, s>>>(counts, offsets, bsums, T);
    scan_sums_kernel<<<1, 1024, 0, s>>>(bsums, nblk, offsets + T);
    scan_add_kernel<<<nblk, 1024, 0, s>>>(offsets, cursor, bsums, T);
    {
      ProfScope ps("msm_scatter", s, nd, nd * 32 + (double)entries * 4);
      msm_scatter_kernel<<<g, 256, 0, s>>>(d_scalars, n, (uint32_t)p.c, Wj, cursor, list, job_off, jobs);
    }
    nl += 5;
    {
      // convention: 6 Fq products per point-window (the batch-affine cost);
      // algorithmic bytes: each entry's index and signed base read once
      ProfScope ps("msm_bucket", s, (double)entries * 6, (double)entries * 68);
      ba_setup_kernel<<<gb, 256, 0, s>>>(counts, offsets, list, bases, cnt, fin, T);
      nl++;
      uint64_t jb = l.jb[0];
      for (uint32_t r = 0; r < l.rounds; r++) {
        const bool first = r == 0;
        uint32_t* jo = joff[r & 1];
        const uint32_t* in_off = first ? offsets : joff[(r + 1) & 1];
        const fe* src = first ? bases : buf[(r + 1) & 1];
        fe* dst = buf[r & 1];
        ba_jobs_kernel<<<gb, 256, 0, s>>>(cnt, cprev, np, T);
        scan_block_kernel<<<nblk, 1024, 0, s>>>(np, jo, bsums, T);
        scan_sums_kernel<<<1, 1024, 0, s>>>(bsums, nblk, jo + T);
        scan_add_kernel<<<nblk, 1024, 0, s>>>(jo, cursor, bsums, T);
        // inversion threads: enough to fill the GPU (fill groups), each group
        // at most BA_G task products; the grid covers the one-task groups of
        // a small round
        const uint64_t tasks = ba_tasks_bound(jb, fill_k);
        const uint32_t fill = (uint32_t)sms * 32;
        const unsigned gt = (unsigned)std::min<uint64_t>((tasks + 255) / 256, (uint64_t)sms * 6);
        const uint64_t groups = tasks < fill ? tasks : std::max<uint64_t>(2ull * fill, tasks / BA_G + 1);
        const unsigned gi = (unsigned)std::min<uint64_t>((groups + 127) / 128, (uint64_t)sms * 8);
        if (first)
          ba_prefix_kernel<true><<<gt, 256, kPrefixSmem, s>>>(src, list, in_off, cprev, jo, T, pre, tot, fill_k);
        else
          ba_prefix_kernel<false><<<gt, 256, kPrefixSmem, s>>>(src, list, in_off, cprev, jo, T, pre, tot, fill_k);
        ba_invert_kernel<<<gi, 128, 0, s>>>(tot, tpre, jo, T, fill, fill_k);
        if (first)
          ba_apply_kernel<true><<<gt, 256, kApplySmem, s>>>(src, list, in_off, cprev, jo, np, T, pre, tot, dst, fin,
                                                            cnt, fill_k);
        else
          ba_apply_kernel<false><<<gt, 256, kApplySmem, s>>>(src, list, in_off, cprev, jo, np, T, pre, tot, dst, fin,
                                                             cnt, fill_k);
        nl += 7;
        jb = jb / 2 + T;
      }
      // tail: chunk counts -> scan (offsets in joff of the unused parity) -> folds -> bucket sums
      const uint32_t last = (l.rounds - 1) & 1;
      uint32_t* coff = joff[last ^ 1];
      ba_chunks_kernel<<<gb, 256, 0, s>>>(cnt, nch, T);
      scan_block_kernel<<<nblk, 1024, 0, s>>>(nch, coff, bsums, T);
      scan_sums_kernel<<<1, 1024, 0, s>>>(bsums, nblk, coff + T);
      scan_add_kernel<<<nblk, 1024, 0, s>>>(coff, cursor, bsums, T);
      cudaMemsetAsync(heavy_count, 0, 4, s);
      const unsigned gf = (unsigned)std::min<uint64_t>((l.chunks + 255) / 256, (uint64_t)sms * 8);
      ba_fold_kernel<<<gf, 256, 0, s>>>(cnt, joff[last], buf[last], fin, coff, nch, T, chunk_res);
      ba_bucket_sum_kernel<<<gb, 256, 0, s>>>(coff, nch, chunk_res, buckets, heavy, heavy_count, T);
      const uint64_t max_heavy = std::min<uint64_t>(T, l.chunks / (BA_TSEQ + 1) + 1);
      ba_heavy_kernel<<<(unsigned)max_heavy, 256, 0, s>>>(coff, nch, chunk_res, buckets, heavy, heavy_count);
      nl += 8;
    }
    {
      ProfScope ps("msm_segment", s, (double)T * 2 * 14, T * 128.0);
      msm_segment_kernel<<<(segs + 127) / 128, 128, 0, s>>>(buckets, segres, segsum, B, L, segs);
    }
    msm_window_kernel<<<W, 256, kWindowSmem, s>>>(segres, segsum, winsum, B / L, L);
    nl += 2;
    e = cudaGetLastError();
    if (!wout && e == cudaSuccess) e = horner_on_host(winsum, W, (uint32_t)p.c, d_out, s);
  }
  for (void* ptr : {(void*)counts, (void*)offsets, (void*)cursor, (void*)bsums, (void*)list, (void*)cnt,
                    (void*)cprev, (void*)np, (void*)joff[0], (void*)joff[1], (void*)fin, (void*)buf[0],
                    (void*)buf[1], (void*)pre, (void*)tot, (void*)tpre, (void*)buckets, (void*)segres, (void*)segsum,
                    (void*)nch, (void*)heavy, (void*)heavy_count, (void*)chunk_res,
                    (void*)(wout ? nullptr : winsum), (void*)bases_rp})
    if (ptr) cudaFreeAsync(ptr, s);
  if (launches) *launches = nl;
  return e;
}
}  // namespace

uint64_t msm_scratch_bytes(uint64_t n_total, uint32_t jobs, uint64_t nbases, bool bases_rp_given, bool own_winsum,
                           int device) {
  if (n_total == 0) return 256;
  const MsmLayout l = msm_layout(n_total, jobs, 0, device);
  if (!l.ok) return ~0ull >> 2;
  return l.bytes(own_winsum, bases_rp_given ? 0 : nbases);
}

cudaError_t msm_convert_bases(const fe* d_in, fe* d_out, uint64_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  msm_convert_bases_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_in, d_out, n);
  return cudaGetLastError();
}

cudaError_t msm_run(const fe* d_scalars, const fe* d_bases, uint64_t n, fe* d_out, cudaStream_t s, int c_override,
                    uint64_t* launches, MsmWindowsOut* wout, bool bases_rp) {
  return msm_run_impl(d_scalars, d_bases, n, d_out, s, c_override, launches, wout, nullptr, 1, n, bases_rp);
}

cudaError_t msm_run_multi(const fe* d_scalars, const fe* d_bases, const uint32_t* d_job_off, uint32_t jobs,
                          uint64_t n_total, uint64_t max_n, cudaStream_t s, uint64_t* launches, MsmWindowsOut* wout,
                          bool bases_rp) {
  if (!wout || !wout->d_winsum || jobs == 0 || !d_job_off || n_total >= (1ull << 32)) return cudaErrorInvalidValue;
  return msm_run_impl(d_scalars, d_bases, n_total, nullptr, s, 0, launches, wout, d_job_off, jobs, max_n, bases_rp);
}

}  // namespace zk
