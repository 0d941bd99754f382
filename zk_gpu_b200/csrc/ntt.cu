// ntt.cu — Fr NTT pass kernels and host orchestration (see ntt.cuh).
//
// Per pass, one CTA owns G columns of one outer block (or, in the last pass,
// G groups whose outputs are adjacent).  Each thread holds 8 elements of one
// column and runs the m-point DIF DFT as "rounds": a round covers three
// index bits [lo, lo+3) that the thread holds in registers and performs the
// radix-2 stages whose butterfly bit falls in that range.  Between rounds the
// column is exchanged through shared memory, stored as 8 u32 planes with the
// XOR swizzle  addr = e ^ ((e >> 3) & 31),  which keeps every round's
// 32-lane access pattern on 32 distinct banks for all b in [3, 12].
// Twiddles of the last round are the 8th roots of unity (compile-time
// indices, broadcast reads); the w == 1 butterflies skip the product.
// Values stay in [0, 2p) between stages (lazy reduction, 4p < 2^256) and
// are made canonical on the final store.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "ntt.cuh"
#include "ntt_tile.cuh"
#include "prof.cuh"
#include "runtime.cuh"

namespace zk {

NttPlan make_ntt_plan(int log_n) {
  NttPlan p;
  p.log_n = log_n;
  if (log_n <= 2) {  // direct DFT kernel
    p.npass = 0;
    return p;
  }
  if (log_n <= 11) {
    p.npass = 1;
    p.bits[0] = log_n;
    return p;
  }
  int np = (log_n + 8) / 9;  // passes of at most 9 bits
  if (np < 2) np = 2;
  p.npass = np;
  int base = log_n / np, extra = log_n % np;
  for (int t = 0; t < np; t++) p.bits[t] = base + (t < extra ? 1 : 0);
  return p;
}


// ---------------------------------------------------------------------------
// persistent batch kernel: the passes of many transforms in one launch
// ---------------------------------------------------------------------------
// Work items are CTA tiles ordered by pass level (every first pass before any
// second pass, ...).  A CTA takes the next item with one atomic; before a
// tile of pass t it waits for all tiles of pass t-1 of the same transform.
// Those were handed out earlier to CTAs that are already running and never
// wait on later items, so the waits always end; each is still bounded by a
// clock budget after which the kernel records an error and stops.
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__global__ void __launch_bounds__(256, 2) ntt_batch_kernel(const BatchPass* passes, uint32_t npass,
                                                          uint32_t total_tiles, uint32_t* next, uint32_t* done,
                                                          uint32_t* err, uint64_t spin_cycles) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ uint32_t s_w, s_k, s_stop;
  for (;;) {
    if (threadIdx.x == 0) {
      uint32_t w = atomicAdd(next, 1u);
      s_stop = (w >= total_tiles || ld_acquire_u32(err) != 0) ? 1u : 0u;
      if (!s_stop) {
        // last pass whose first tile index is <= w
        uint32_t lo = 0, hi = npass;
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) / 2;
          if (passes[mid].tile_base <= w) lo = mid; else hi = mid;
        }
        const BatchPass& bp = passes[lo];
        if (bp.dep != 0xffffffffu) {
          const uint64_t t0 = clock64();
          while (ld_acquire_u32(done + bp.dep) < bp.dep_tiles) {
            if (clock64() - t0 > spin_cycles) {
              atomicExch(err, 1u);
              s_stop = 1;
              break;
            }
            __nanosleep(64);
          }
        }
        s_w = w;
        s_k = lo;
      }
    }
    __syncthreads();
    if (s_stop) return;
    const BatchPass& bp = passes[s_k];
    const uint64_t tile = s_w - bp.tile_base;
    switch (bp.B) {
      case 3: ntt_pass_tile<3, true>(bp.p, tile, smem); break;
      case 4: ntt_pass_tile<4, true>(bp.p, tile, smem); break;
      case 5: ntt_pass_tile<5, true>(bp.p, tile, smem); break;
      case 6: ntt_pass_tile<6, true>(bp.p, tile, smem); break;
      case 7: ntt_pass_tile<7, true>(bp.p, tile, smem); break;
      case 8: ntt_pass_tile<8, true>(bp.p, tile, smem); break;
      case 9: ntt_pass_tile<9, true>(bp.p, tile, smem); break;
      case 10: ntt_pass_tile<10, true>(bp.p, tile, smem); break;
      case 11: ntt_pass_tile<11, true>(bp.p, tile, smem); break;
      default: break;
    }
    __threadfence();  // every thread publishes its own stores before the tile is counted
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(done + s_k, 1u);
    }
  }
}

// Tiny transforms (n <= 4): direct DFT, one thread per output.
__global__ void ntt_tiny_kernel(fe* a, uint32_t log_n, fe w, const fe* pre_lo, const fe* pre_hi, uint32_t pre_shift,
                                uint32_t has_post, fe post) {
  const uint32_t n = 1u << log_n;
  const uint32_t k = threadIdx.x;
  uint32_t in[4][8];
  for (uint32_t i = 0; i < n; i++) {
    ld_fe(in[i], a + i);
    if (pre_lo) {
      uint32_t c0[8], c1[8];
      ld_fe_nc(c0, pre_lo + (i & ((1u << pre_shift) - 1)));
      ld_fe_nc(c1, pre_hi + (i >> pre_shift));
      mul_rp<P_r>(c0, c0, c1);
      mul_rp<P_r>(in[i], in[i], c0);
      reduce_once<P_r>(in[i], in[i]);
    }
  }
  uint32_t acc[8];
  if (k < n) {
    uint32_t wk[8], wik[8];
    pow_u64<P_r>(wk, w.w, k);
    set_zero(acc);
    set_one<P_r>(wik);
    for (uint32_t i = 0; i < n; i++) {
      uint32_t t[8];
      mul<P_r>(t, in[i], wik);
      add<P_r>(acc, acc, t);
      mul<P_r>(wik, wik, wk);
    }
    if (has_post) {
      mul_rp<P_r>(acc, acc, post.w);
      reduce_once<P_r>(acc, acc);
    }
  }
  __syncthreads();
  if (k < n) st_fe(a + k, acc);
}

// out[e] = base^(e) for e < count (per-thread square-and-multiply)
__global__ void pow_seq_kernel(fe* out, fe base, uint64_t count, uint64_t step) {
  const uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (e >= count) return;
  uint32_t r[8];
  pow_u64_rp<P_r>(r, base.w, e * step);
  st_fe(out + e, r);
}

// twist[k * J + j] = lo[(k j) & mask] * hi[(k j) >> shift]
__global__ void twist_table_kernel(fe* out, const fe* lo, const fe* hi, uint32_t shift, uint32_t log_J, uint64_t total) {
  const uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const uint64_t k = idx >> log_J, j = idx & ((1ull << log_J) - 1);
  const uint64_t e = k * j;
  uint32_t a[8], b[8];
  ld_fe_nc(a, lo + (e & ((1ull << shift) - 1)));
  ld_fe_nc(b, hi + (e >> shift));
  mul_rp<P_r>(a, a, b);
  reduce_once<P_r>(a, a);
  st_fe(out + idx, a);
}

// dst[i * dst_stride] = src[i] * c^i (powc may be null: plain strided copy)
__global__ void scale_copy_kernel(fe* dst, const fe* src, uint64_t n, uint64_t dst_stride, const fe* lo, const fe* hi,
                                  uint32_t shift) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t v[8];
  ld_fe(v, src + i);
  if (lo) {
    uint32_t a[8], b[8];
    ld_fe_nc(a, lo + (i & ((1ull << shift) - 1)));
    ld_fe_nc(b, hi + (i >> shift));
    mul_rp<P_r>(a, a, b);
    mul_rp<P_r>(v, v, a);
    reduce_once<P_r>(v, v);
  }
  st_fe(dst + i * dst_stride, v);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static fe to_fe(const host::Fr& a) {
  fe r;
  std::memcpy(r.w, a.v, 32);
  return r;
}
// R-form (x 2^256) -> R'-form (x 2^260): every constant the kernels multiply
// data by (roots, twists, coset powers, scales) is kept in R' form for mul_rp.
static fe to_fe_rp(const host::Fr& a) { return to_fe(host::mul(a, host::from_u64(16))); }

static cudaError_t pow_two_level(fe** lo, fe** hi, uint32_t* shift, const host::Fr& base, int log_count,
                                 cudaStream_t s, bool pooled) {
  const uint32_t sh = (uint32_t)((log_count + 1) / 2);
  const uint64_t nlo = 1ull << sh, nhi = 1ull << (log_count > (int)sh ? log_count - sh : 0);
  cudaError_t e;
  *lo = *hi = nullptr;
  if (pooled) {
    e = zk::dmalloc((void**)lo, nlo * sizeof(fe), s);
    if (e != cudaSuccess) return e;
    e = zk::dmalloc((void**)hi, nhi * sizeof(fe), s);
    if (e != cudaSuccess) return e;
  } else {
    e = cudaMalloc((void**)lo, nlo * sizeof(fe));
    if (e != cudaSuccess) return e;
    e = cudaMalloc((void**)hi, nhi * sizeof(fe));
    if (e != cudaSuccess) return e;
  }
  const host::Fr bstep = host::pow_2k(base, sh);
  pow_seq_kernel<<<(unsigned)((nlo + 255) / 256), 256, 0, s>>>(*lo, to_fe_rp(base), nlo, 1);
  pow_seq_kernel<<<(unsigned)((nhi + 255) / 256), 256, 0, s>>>(*hi, to_fe_rp(bstep), nhi, 1);
  *shift = sh;
  return cudaGetLastError();
}

// t[i] *= scale (R' form)
__global__ void scale_table_kernel(fe* t, fe scale, uint64_t count) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t v[8];
  ld_fe(v, t + i);
  mul_rp<P_r>(v, v, scale.w);
  reduce_once<P_r>(v, v);
  st_fe(t + i, v);
}

cudaError_t pow_tables_make(PowTables* t, const host::Fr& c, int log_n, cudaStream_t s, const host::Fr* scale,
                            bool pooled) {
  cudaError_t e = pow_two_level(&t->lo, &t->hi, &t->shift, c, log_n, s, pooled);
  if (e == cudaSuccess && scale) {
    const uint64_t nlo = 1ull << t->shift;
    scale_table_kernel<<<(unsigned)((nlo + 255) / 256), 256, 0, s>>>(t->lo, to_fe_rp(*scale), nlo);
    e = cudaGetLastError();
  }
  return e;
}
void pow_tables_free(PowTables* t, cudaStream_t s) {
  if (t->lo) cudaFreeAsync(t->lo, s);
  if (t->hi) cudaFreeAsync(t->hi, s);
  t->lo = t->hi = nullptr;
}

static cudaError_t build_tables(NttTables* t, cudaStream_t s) {
  const NttPlan& p = t->plan;
  int done_bits = 0;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < p.npass; k++) {
    const int b = p.bits[k];
    const int log_J = p.log_n - done_bits - b;  // later passes' bits
    // this pass works on the sub-problem of size m*J whose root is w^(n / (m J))
    const host::Fr wMJ = host::pow_2k(t->omega, (unsigned)done_bits);
    const host::Fr wm = host::pow_2k(wMJ, (unsigned)log_J);
    const uint64_t half = b >= 1 ? (1ull << (b - 1)) : 1;
    e = cudaMalloc((void**)&t->inner[k], half * sizeof(fe));
    if (e != cudaSuccess) return e;
    t->bytes += half * sizeof(fe);
    pow_seq_kernel<<<(unsigned)((half + 255) / 256), 256, 0, s>>>(t->inner[k], to_fe_rp(wm), half, 1);
    if (k + 1 < p.npass) {
      const uint64_t total = 1ull << (b + log_J);
      e = cudaMalloc((void**)&t->twist[k], total * sizeof(fe));
      if (e != cudaSuccess) return e;
      t->bytes += total * sizeof(fe);
      fe *lo = nullptr, *hi = nullptr;
      uint32_t sh = 0;
      e = pow_two_level(&lo, &hi, &sh, wMJ, b + log_J, s, true);
      if (e != cudaSuccess) return e;
      twist_table_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(t->twist[k], lo, hi, sh, (uint32_t)log_J, total);
      cudaFreeAsync(lo, s);
      cudaFreeAsync(hi, s);
    }
    done_bits += b;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}

size_t ntt_tables_elems(int log_n) {
  const NttPlan p = make_ntt_plan(log_n);
  size_t total = 0;
  int done = 0;
  for (int k = 0; k < p.npass; k++) {
    const int b = p.bits[k];
    const int log_J = p.log_n - done - b;
    total += b >= 1 ? (1ull << (b - 1)) : 1;
    if (k + 1 < p.npass) {
      const int lc = b + log_J;
      const int sh = (lc + 1) / 2;
      total += (1ull << lc) + (1ull << sh) + (1ull << (lc > sh ? lc - sh : 0));
    }
    done += b;
  }
  return total;
}

cudaError_t ntt_tables_fill(NttTables* t, const host::Fr& omega, int log_n, fe* mem, size_t cap, cudaStream_t s) {
  if (ntt_tables_elems(log_n) > cap) return cudaErrorInvalidValue;
  t->plan = make_ntt_plan(log_n);
  t->omega = omega;
  t->bytes = 0;
  const NttPlan& p = t->plan;
  fe* cur = mem;
  int done = 0;
  for (int k = 0; k < p.npass; k++) {
    const int b = p.bits[k];
    const int log_J = p.log_n - done - b;
    const host::Fr wMJ = host::pow_2k(omega, (unsigned)done);
    const host::Fr wm = host::pow_2k(wMJ, (unsigned)log_J);
    const uint64_t half = b >= 1 ? (1ull << (b - 1)) : 1;
    t->inner[k] = cur;
    cur += half;
    pow_seq_kernel<<<(unsigned)((half + 255) / 256), 256, 0, s>>>(t->inner[k], to_fe_rp(wm), half, 1);
    if (k + 1 < p.npass) {
      const int lc = b + log_J;
      const uint32_t sh = (uint32_t)((lc + 1) / 2);
      const uint64_t total = 1ull << lc, nlo = 1ull << sh, nhi = 1ull << (lc > (int)sh ? lc - sh : 0);
      fe* lo = cur;
      fe* hi = cur + nlo;
      t->twist[k] = cur + nlo + nhi;
      cur += nlo + nhi + total;
      pow_seq_kernel<<<(unsigned)((nlo + 255) / 256), 256, 0, s>>>(lo, to_fe_rp(wMJ), nlo, 1);
      pow_seq_kernel<<<(unsigned)((nhi + 255) / 256), 256, 0, s>>>(hi, to_fe_rp(host::pow_2k(wMJ, sh)), nhi, 1);
      twist_table_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(t->twist[k], lo, hi, sh, (uint32_t)log_J,
                                                                          total);
    } else {
      t->twist[k] = nullptr;
    }
    done += b;
  }
  return cudaGetLastError();
}

bool ntt_plan_valid(const NttPlan& p) {
  if (p.log_n < 0 || p.log_n > NTT_MAX_LOG) return false;
  if (p.log_n <= 2) return p.npass == 0;
  if (p.npass < 1 || p.npass > NTT_MAX_PASS) return false;
  if (p.npass == 1) return p.bits[0] == p.log_n && p.log_n <= 11;
  int sum = 0;
  for (int k = 0; k < p.npass; k++) {
    if (p.bits[k] < 3 || p.bits[k] > 11) return false;
    sum += p.bits[k];
  }
  for (int k = p.npass; k < NTT_MAX_PASS; k++)
    if (p.bits[k] != 0) return false;
  return sum == p.log_n;
}

cudaError_t ntt_tables_build(NttTables* t, const NttPlan& plan, const host::Fr& omega, cudaStream_t s) {
  if (!ntt_plan_valid(plan)) return cudaErrorInvalidValue;
  *t = NttTables{};
  t->plan = plan;
  t->omega = omega;
  cudaError_t e = build_tables(t, s);
  if (e != cudaSuccess) ntt_tables_release(t);
  return e;
}

void ntt_tables_release(NttTables* t) {
  for (int k = 0; k < NTT_MAX_PASS; k++) {
    if (t->inner[k]) cudaFree(t->inner[k]);
    if (t->twist[k]) cudaFree(t->twist[k]);
    t->inner[k] = t->twist[k] = nullptr;
  }
  t->bytes = 0;
}

static cudaError_t dispatch_pass(int B, const PassParams& pp, uint64_t ncta, cudaStream_t s) {
  switch (B) {
    case 3: return launch_pass<3>(pp, ncta, s);
    case 4: return launch_pass<4>(pp, ncta, s);
    case 5: return launch_pass<5>(pp, ncta, s);
    case 6: return launch_pass<6>(pp, ncta, s);
    case 7: case 8: case 9: case 10: case 11: return launch_pass_wide(B, pp, ncta, s);
    default: return cudaErrorInvalidValue;
  }
}

uint64_t ntt_pass_params(const NttTables& t, int k, fe* d_a, fe* d_tmp, const PowTables* pre, const host::Fr* post,
                         PassParams* out) {
  NttFuse f;
  f.pre = pre;
  f.post = post;
  return ntt_pass_params(t, k, d_a, d_tmp, f, out);
}

uint64_t ntt_pass_params(const NttTables& t, int k, fe* d_a, fe* d_tmp, const NttFuse& f, PassParams* out) {
  const PowTables* pre = f.pre;
  const host::Fr* post = f.post;
  const NttPlan& p = t.plan;
  const int L = p.log_n;
  int done = 0;
  for (int j = 0; j < k; j++) done += p.bits[j];
  const int b = p.bits[k];
  const bool final_pass = (k + 1 == p.npass);
  PassParams pp{};
  pp.inner = t.inner[k];
  pp.twist = t.twist[k];
  pp.log_J = (uint32_t)(L - done - b);
  pp.log_O = (uint32_t)done;
  // final-pass grouping runs over consecutive first digits k_1; a single-pass
  // plan has no digits (one group, rest_count = 1)
  pp.log_m1 = p.npass > 1 ? (uint32_t)p.bits[0] : 0u;
  pp.nprev = final_pass ? (uint32_t)k : 0u;
  for (int j = 0; j < k && j < NTT_MAX_PASS; j++) pp.prev_bits[j] = (uint32_t)p.bits[j];
  pp.is_final = final_pass ? 1u : 0u;
  if (k == 0 && pre) {
    pp.pre_lo = pre->lo;
    pp.pre_hi = pre->hi;
    pp.pre_shift = pre->shift;
  }
  if (final_pass && post) {
    pp.has_post = 1;
    pp.post = to_fe_rp(*post);
  }
  if (final_pass && f.post_tab) {
    pp.post_lo = f.post_tab->lo;
    pp.post_hi = f.post_tab->hi;
    pp.post_shift = f.post_tab->shift;
  }
  if (k == 0 && f.nonzero) {
    // first pass reads rows of J = 2^(L - b) elements: whole zero rows are skipped
    const uint64_t J = 1ull << (L - b);
    if (f.nonzero % J == 0 && f.nonzero / J < (1ull << b)) pp.in_rows = (uint32_t)(f.nonzero / J);
  }
  // buffers: single pass in place; otherwise a -> tmp, tmp in place, tmp -> a
  if (p.npass == 1) {
    pp.in = d_a;
    pp.out = d_a;
  } else if (k == 0) {
    pp.in = d_a;
    pp.out = d_tmp;
  } else if (!final_pass) {
    pp.in = d_tmp;
    pp.out = d_tmp;
  } else {
    pp.in = d_tmp;
    pp.out = d_a;
  }
  if (k == 0 && f.src) pp.in = f.src;  // out of place: the first pass reads the source
  const uint32_t Gmax = b >= 11 ? 1u : (1u << (11 - b));
  uint64_t groups_dim;
  if (!final_pass) {
    groups_dim = 1ull << pp.log_J;  // columns per outer block
  } else if (p.npass == 1) {
    groups_dim = 1;
  } else {
    groups_dim = 1ull << p.bits[0];  // consecutive k_1 digits
  }
  pp.G = (uint32_t)std::min<uint64_t>(Gmax, groups_dim);
  *out = pp;
  return (1ull << (L - b)) / pp.G;
}

cudaError_t ntt_run(const NttTables& t, fe* d_a, fe* d_tmp, const PowTables* pre, const host::Fr* post, cudaStream_t s) {
  NttFuse f;
  f.pre = pre;
  f.post = post;
  return ntt_run(t, d_a, d_tmp, f, s);
}

cudaError_t ntt_run(const NttTables& t, fe* d_a, fe* d_tmp, const NttFuse& f, cudaStream_t s) {
  const PowTables* pre = f.pre;
  const host::Fr* post = f.post;
  const NttPlan& p = t.plan;
  const int L = p.log_n;
  if (L <= 2) {
    if (f.post_tab) return cudaErrorInvalidValue;  // the direct kernel takes constant scales only
    fe po{};
    if (post) po = to_fe_rp(*post);
    ntt_tiny_kernel<<<1, 32, 0, s>>>(d_a, (uint32_t)L, to_fe(t.omega), pre ? pre->lo : nullptr, pre ? pre->hi : nullptr,
                                     pre ? pre->shift : 0u, post ? 1u : 0u, po);
    return cudaGetLastError();
  }
  static const char* names[12] = {"", "", "", "ntt_pass_b3", "ntt_pass_b4", "ntt_pass_b5", "ntt_pass_b6",
                                  "ntt_pass_b7", "ntt_pass_b8", "ntt_pass_b9", "ntt_pass_b10", "ntt_pass_b11"};
  for (int k = 0; k < p.npass; k++) {
    const int b = p.bits[k];
    PassParams pp;
    const uint64_t ncta = ntt_pass_params(t, k, d_a, d_tmp, f, &pp);
    const double nel = (double)(1ull << L);
    // algorithmic work: radix-2 convention (n/2) * b products; bytes: read + write (+ twist table)
    ProfScope prof(names[b], s, nel / 2 * b, nel * 32.0 * (pp.is_final ? 2 : 3));
    cudaError_t e = dispatch_pass(b, pp, ncta, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static size_t batch_smem_bytes() { return (size_t)8 * 2048 * 4 + (size_t)1024 * 40; }  // B <= 11

int ntt_batch_grid(int device) {
  static int cached[64] = {0};
  if (device >= 0 && device < 64 && cached[device]) return cached[device];
  cudaFuncSetAttribute(ntt_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batch_smem_bytes());
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ntt_batch_kernel, 256, batch_smem_bytes());
  const int g = sms * (per_sm > 0 ? per_sm : 1);
  if (device >= 0 && device < 64) cached[device] = g;
  return g;
}

cudaError_t ntt_batch_launch(const BatchPass* d_passes, uint32_t npass, uint32_t total_tiles, uint32_t* d_next,
                             uint32_t* d_done, uint32_t* d_err, int grid, cudaStream_t s, uint64_t spin_cycles) {
  ntt_batch_kernel<<<grid, 256, batch_smem_bytes(), s>>>(d_passes, npass, total_tiles, d_next, d_done, d_err,
                                                         spin_cycles);
  return cudaGetLastError();
}

cudaError_t fr_scale_copy(fe* dst, const fe* src, size_t n, size_t dst_stride, const PowTables* powc, cudaStream_t s) {
  scale_copy_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dst, src, n, dst_stride, powc ? powc->lo : nullptr,
                                                               powc ? powc->hi : nullptr, powc ? powc->shift : 0);
  return cudaGetLastError();
}

}  // namespace zk
