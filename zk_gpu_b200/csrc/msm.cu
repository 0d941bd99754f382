// msm.cu — Pippenger MSM kernels and orchestration (see msm.cuh).
#include <algorithm>

#include "curve.cuh"
#include "msm.cuh"
#include "prof.cuh"

namespace zk {

MsmPlan make_msm_plan(uint64_t n, int c_override) {
  MsmPlan p;
  int lg = 1;
  while ((1ull << lg) < n) lg++;
  int c = lg - 4;
  if (c < 4) c = 4;
  if (c > 16) c = 16;
  if (c_override == 0) {  // the autotuner's choice for this device and size, if any
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) c_override = tuned_msm_window(dev, lg);
  }
  if (c_override >= 3 && c_override <= 20) c = c_override;
  p.c = c;
  p.windows = (254 + c - 1) / c;
  p.buckets = 1u << (c - 1);
  // buckets per reduction segment: each segment thread's latency is its
  // running sum (2L additions) plus the weight multiply lo * S (about c
  // doublings).  Few buckets per window: short segments (L = 4) for
  // parallelism; many (2^12 and up): L = 16, since the extra weight
  // multiplies of 4x more segments cost more than they save (measured on
  // B200: 2^14 points, c = 10: 0.57 -> 0.24 ms; 2^22, c = 15: 0.9 -> 1.6 ms)
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

// Buckets are split into sub-buckets of at most SUB entries, one thread
// each, so a bucket that collects a large share of the points (skewed
// scalars, e.g. many small ones all carrying into the same digit) is summed
// by many threads instead of one.
constexpr uint32_t SUB_MAX = 64;      // entries per sub-bucket (large MSMs)
constexpr uint32_t SUB_MIN = 16;      // small MSMs: shorter chains, more threads
constexpr uint32_t SEQ_MAX = 16;      // sub-sums a bucket combines in one thread

__global__ void msm_nsub_kernel(const uint32_t* counts, uint32_t* nsub, uint32_t total, uint32_t sub_len) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < total) nsub[b] = (counts[b] + sub_len - 1) / sub_len;
}

__global__ void msm_submap_kernel(const uint32_t* nsub, const uint32_t* sub_off, uint32_t* sub2b, uint32_t total) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= total) return;
  const uint32_t k = nsub[b], o = sub_off[b];
  for (uint32_t j = 0; j < k; j++) sub2b[o + j] = b;
}

// One thread per sub-bucket: sum of its (signed) points.
__global__ void __launch_bounds__(256) msm_subbucket_kernel(const uint32_t* list, const uint32_t* offsets,
                                                            const uint32_t* counts, const uint32_t* sub_off,
                                                            const uint32_t* sub2b, const uint32_t* total_sub,
                                                            const fe* bases, fe* subres, uint32_t sub_len) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= *total_sub) return;
  const uint32_t b = sub2b[s];
  const uint32_t j = s - sub_off[b];
  const uint32_t beg = offsets[b] + j * sub_len;
  const uint32_t end = min(offsets[b] + counts[b], beg + sub_len);
  xyzz_t acc;
  xyzz_set_inf(acc);
  for (uint32_t k = beg; k < end; k++) {
    const uint32_t e = list[k];
    aff_t q;
    ld_aff(q, bases + 2 * (uint64_t)(e & 0x7fffffffu));
    if (aff_is_inf(q)) continue;
    if (e & 0x80000000u) {
      uint32_t z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      sub<FqP>(q.y, z, q.y);
    }
    xyzz_madd(acc, q);
  }
  st_xyzz(subres + 4 * (uint64_t)s, acc);
}

// One thread per bucket: combine its sub-sums when there are few; queue the
// bucket for the block-wide reduction when there are many.
__global__ void msm_bucket_final_kernel(const uint32_t* nsub, const uint32_t* sub_off, const fe* subres, fe* buckets,
                                        uint32_t* heavy, uint32_t* heavy_count, uint32_t total) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= total) return;
  const uint32_t k = nsub[b], o = sub_off[b];
  if (k > SEQ_MAX) {
    heavy[atomicAdd(heavy_count, 1u)] = b;
    return;
  }
  xyzz_t acc, t;
  xyzz_set_inf(acc);
  for (uint32_t j = 0; j < k; j++) {
    ld_xyzz(t, subres + 4 * (uint64_t)(o + j));
    xyzz_add(acc, t);
  }
  st_xyzz(buckets + 4 * (uint64_t)b, acc);
}

// One block per queued heavy bucket: strided partial sums, then a tree.
__global__ void __launch_bounds__(256) msm_heavy_kernel(const uint32_t* nsub, const uint32_t* sub_off,
                                                        const fe* subres, fe* buckets, const uint32_t* heavy,
                                                        const uint32_t* heavy_count) {
  __shared__ fe sh[256 * 4];
  if (blockIdx.x >= *heavy_count) return;
  const uint32_t b = heavy[blockIdx.x];
  const uint32_t k = nsub[b], o = sub_off[b];
  xyzz_t acc, t;
  xyzz_set_inf(acc);
  for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
    ld_xyzz(t, subres + 4 * (uint64_t)(o + j));
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

// Per (window, segment): running sums over the segment's buckets, top down,
// giving sum_j (j - lo + 1) B_j and sum_j B_j; result T + lo * S, which is
// the segment's share of sum_j (j + 1) B_j.
__global__ void __launch_bounds__(128) msm_segment_kernel(const fe* buckets, fe* segres, uint32_t B, uint32_t L,
                                                          uint32_t total_segs) {
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
  xyzz_mul_small(run, lo);
  xyzz_add(tot, run);
  st_xyzz(segres + 4 * (uint64_t)gs, tot);
}

// One block per window: tree sum of its segment results.
__global__ void __launch_bounds__(256) msm_window_kernel(const fe* segres, fe* winsum, uint32_t S_per_w) {
  __shared__ fe sh[256 * 4];
  const uint32_t w = blockIdx.x;
  xyzz_t acc, t;
  xyzz_set_inf(acc);
  for (uint32_t s = threadIdx.x; s < S_per_w; s += blockDim.x) {
    ld_xyzz(t, segres + 4 * ((uint64_t)w * S_per_w + s));
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
    st_xyzz(winsum + 4 * (uint64_t)w, acc);
  }
}

// Horner over windows (high to low) and conversion to Jacobian.
__global__ void msm_combine_kernel(const fe* winsum, uint32_t windows, uint32_t c, fe* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  xyzz_t acc, t;
  ld_xyzz(acc, winsum + 4 * (uint64_t)(windows - 1));
  for (int w = (int)windows - 2; w >= 0; w--) {
    for (uint32_t k = 0; k < c; k++) xyzz_dbl(acc, acc);
    ld_xyzz(t, winsum + 4 * (uint64_t)w);
    xyzz_add(acc, t);
  }
  uint32_t j[24];
  xyzz_to_jacobian(j, acc);
  st_fe(out, j);
  st_fe(out + 1, j + 8);
  st_fe(out + 2, j + 16);
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
// n: scalars (all jobs); jobs > 1: job_off (device, jobs + 1 entries) splits
// them and every job reads bases [0, nbases); the window sums of job j are
// windows [j W, (j + 1) W) of wout.
cudaError_t msm_run_impl(const fe* d_scalars, const fe* d_bases, uint64_t n, fe* d_out, cudaStream_t s,
                         int c_override, uint64_t* launches, MsmWindowsOut* wout, const uint32_t* job_off,
                         uint32_t jobs, uint64_t nbases) {
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
  // one window size for every job: the plan of the mean job size
  const MsmPlan p = make_msm_plan((n + jobs - 1) / jobs, c_override);
  if (wout) {
    if ((uint32_t)p.windows > MSM_MAX_WINDOWS || !wout->d_winsum) return cudaErrorInvalidValue;
    wout->windows = (uint32_t)p.windows;
    wout->c = (uint32_t)p.c;
  }
  const uint32_t Wj = (uint32_t)p.windows, B = p.buckets, L = p.seg_len;
  const uint32_t W = Wj * jobs;  // windows of all jobs
  if ((uint64_t)W * B >= (1ull << 31)) return cudaErrorInvalidValue;
  const uint32_t total = W * B;
  const uint32_t nblk = (total + 1023) / 1024;
  const uint64_t entries = n * (uint64_t)Wj;
  if (entries >= (1ull << 32)) return cudaErrorInvalidValue;  // entry offsets are 32-bit
  uint32_t *counts = nullptr, *offsets = nullptr, *cursor = nullptr, *bsums = nullptr, *list = nullptr;
  uint32_t *nsub = nullptr, *sub_off = nullptr, *sub2b = nullptr, *heavy = nullptr, *heavy_count = nullptr;
  fe *buckets = nullptr, *segres = nullptr, *winsum = nullptr, *subres = nullptr, *bases_rp = nullptr;
  const uint32_t segs = total / L;
  // sub-bucket size: enough sub-buckets to fill the GPU (about 2^17 threads)
  uint32_t sub_len = SUB_MAX;
  while (sub_len > SUB_MIN && entries / sub_len < (1ull << 17)) sub_len >>= 1;
  // sum_b ceil(count_b / sub_len) <= entries / sub_len + total; heavy buckets have > SEQ_MAX * sub_len entries
  const uint64_t max_sub = entries / sub_len + total + 1;
  const uint64_t max_heavy = entries / ((uint64_t)SEQ_MAX * sub_len) + 1;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** ptr, size_t bytes) {
    if (e == cudaSuccess) e = cudaMallocAsync(ptr, bytes, s);
  };
  alloc((void**)&counts, total * 4ull);
  alloc((void**)&offsets, (total + 1) * 4ull);
  alloc((void**)&cursor, total * 4ull);
  alloc((void**)&bsums, (nblk + 1) * 4ull);
  alloc((void**)&list, entries * 4ull);
  alloc((void**)&nsub, total * 4ull);
  alloc((void**)&sub_off, (total + 1) * 4ull);
  alloc((void**)&sub2b, max_sub * 4ull);
  alloc((void**)&heavy, max_heavy * 4ull);
  alloc((void**)&heavy_count, 4ull);
  alloc((void**)&subres, max_sub * 128ull);
  alloc((void**)&buckets, total * 128ull);
  alloc((void**)&segres, segs * 128ull);
  if (wout)
    winsum = wout->d_winsum;  // caller's buffer, left for the host's Horner step
  else
    alloc((void**)&winsum, W * 128ull);
  alloc((void**)&bases_rp, nbases * 64ull);
  if (e == cudaSuccess) {
    const double nd = (double)n;
    cudaMemsetAsync(counts, 0, total * 4ull, s);
    cudaMemsetAsync(heavy_count, 0, 4ull, s);
    const unsigned g = (unsigned)((n + 255) / 256);
    const unsigned gb = (total + 255) / 256;
    msm_convert_bases_kernel<<<(unsigned)((nbases + 255) / 256), 256, 0, s>>>(d_bases, bases_rp, nbases);
    {
      ProfScope ps("msm_count", s, nd, nd * 32);
      msm_count_kernel<<<g, 256, 0, s>>>(d_scalars, n, (uint32_t)p.c, Wj, counts, job_off, jobs);
    }
    scan_block_kernel<<<nblk, 1024, 0, s>>>(counts, offsets, bsums, total);
    scan_sums_kernel<<<1, 1024, 0, s>>>(bsums, nblk, offsets + total);
    scan_add_kernel<<<nblk, 1024, 0, s>>>(offsets, cursor, bsums, total);
    {
      ProfScope ps("msm_scatter", s, nd, nd * 32 + (double)entries * 4);
      msm_scatter_kernel<<<g, 256, 0, s>>>(d_scalars, n, (uint32_t)p.c, Wj, cursor, list, job_off, jobs);
    }
    msm_nsub_kernel<<<gb, 256, 0, s>>>(counts, nsub, total, sub_len);
    scan_block_kernel<<<nblk, 1024, 0, s>>>(nsub, sub_off, bsums, total);
    scan_sums_kernel<<<1, 1024, 0, s>>>(bsums, nblk, sub_off + total);
    scan_add_kernel<<<nblk, 1024, 0, s>>>(sub_off, cursor, bsums, total);
    msm_submap_kernel<<<gb, 256, 0, s>>>(nsub, sub_off, sub2b, total);
    {
      // convention: 6 Fq products per point-window (batch-affine cost)
      ProfScope ps("msm_bucket", s, (double)entries * 6, (double)entries * (64 + 4) + max_sub * 128.0);
      msm_subbucket_kernel<<<(unsigned)((max_sub + 255) / 256), 256, 0, s>>>(list, offsets, counts, sub_off, sub2b,
                                                                              sub_off + total, bases_rp, subres, sub_len);
    }
    {
      ProfScope ps("msm_bucket_final", s, (double)total * 14, total * 256.0);
      msm_bucket_final_kernel<<<gb, 256, 0, s>>>(nsub, sub_off, subres, buckets, heavy, heavy_count, total);
      msm_heavy_kernel<<<(unsigned)max_heavy, 256, 0, s>>>(nsub, sub_off, subres, buckets, heavy, heavy_count);
    }
    {
      ProfScope ps("msm_segment", s, (double)total * 2 * 14, total * 128.0);
      msm_segment_kernel<<<(segs + 127) / 128, 128, 0, s>>>(buckets, segres, B, L, segs);
    }
    msm_window_kernel<<<W, 256, 0, s>>>(segres, winsum, B / L);
    if (!wout) msm_combine_kernel<<<1, 32, 0, s>>>(winsum, W, (uint32_t)p.c, d_out);
    nl = wout ? 16 : 17;
    e = cudaGetLastError();
  }
  for (void* ptr : {(void*)counts, (void*)offsets, (void*)cursor, (void*)bsums, (void*)list, (void*)nsub,
                    (void*)sub_off, (void*)sub2b, (void*)heavy, (void*)heavy_count, (void*)subres, (void*)buckets,
                    (void*)segres, (void*)(wout ? nullptr : winsum), (void*)bases_rp})
    if (ptr) cudaFreeAsync(ptr, s);
  if (launches) *launches = nl;
  return e;
}
}  // namespace

cudaError_t msm_run(const fe* d_scalars, const fe* d_bases, uint64_t n, fe* d_out, cudaStream_t s, int c_override,
                    uint64_t* launches, MsmWindowsOut* wout) {
  return msm_run_impl(d_scalars, d_bases, n, d_out, s, c_override, launches, wout, nullptr, 1, n);
}

cudaError_t msm_run_multi(const fe* d_scalars, const fe* d_bases, const uint32_t* d_job_off, uint32_t jobs,
                          uint64_t n_total, uint64_t max_n, cudaStream_t s, uint64_t* launches, MsmWindowsOut* wout) {
  if (!wout || !wout->d_winsum || jobs == 0 || !d_job_off || n_total >= (1ull << 32)) return cudaErrorInvalidValue;
  return msm_run_impl(d_scalars, d_bases, n_total, nullptr, s, 0, launches, wout, d_job_off, jobs, max_n);
}

}  // namespace zk
