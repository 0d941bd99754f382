// api_ntt.cu — C-ABI entry points for the NTT, the LDE pipeline and the
// field diagnostics (declared in include/zkgpu.h).
#include <cstring>

#include "fq_inv.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

using zk::fe;
namespace hf = zk::host;

namespace {

hf::Fr load_fr(const uint64_t* p) {
  hf::Fr r;
  std::memcpy(r.v, p, 32);
  return r;
}

// Validate an NTT request; returns ZKGPU_OK or ZKGPU_EINVAL.
int check_ntt_args(const void* data, const uint64_t* omega, uint32_t log_n) {
  if (!data || !omega) return ZKGPU_EINVAL;
  if (log_n > (uint32_t)zk::NTT_MAX_LOG) return ZKGPU_EINVAL;
  hf::Fr w = load_fr(omega);
  if (!hf::is_canonical(w) || !hf::is_primitive_root(w, log_n)) return ZKGPU_EINVAL;
  return ZKGPU_OK;
}

// Enqueue the NTT of d_a (device, in place) with optional coset and scale.
int ntt_device(int device, fe* d_a, uint32_t log_n, const hf::Fr& w, const hf::Fr* coset, const hf::Fr* post,
               cudaStream_t s) {
  (void)device;
  cudaError_t e;
  const zk::NttTablesRef t = zk::ntt_tables_get(device, w, (int)log_n, s, &e);
  if (!t) return zk::status_of("ntt_tables_get", e);
  const size_t n = (size_t)1 << log_n;
  fe* tmp = nullptr;
  if (t->plan.npass > 1) ZK_TRY("zk::dmalloc(ntt scratch)", zk::dmalloc((void**)&tmp, n * sizeof(fe), s));
  zk::PowTables pre;
  if (coset) {
    e = zk::pow_tables_make(&pre, *coset, (int)log_n, s);
    if (e != cudaSuccess) {
      if (tmp) cudaFreeAsync(tmp, s);
      return zk::status_of("pow_tables_make", e);
    }
    zk::count_launches(2);
  }
  e = zk::ntt_run(*t, d_a, tmp, coset ? &pre : nullptr, post, s);
  zk::count_launches(t->plan.npass > 0 ? t->plan.npass : 1);
  if (coset) zk::pow_tables_free(&pre, s);
  if (tmp) cudaFreeAsync(tmp, s);
  return zk::status_of("ntt_run", e);
}

// Host-buffer NTT: upload, transform, download, synchronise.
int ntt_host(int device, uint64_t* a, uint32_t log_n, const uint64_t* omega, const hf::Fr* coset, const hf::Fr* post) {
  int st = check_ntt_args(a, omega, log_n);
  if (st) return st;
  cudaStream_t s;
  st = zk::bind_device(device, &s);
  if (st) return st;
  const size_t bytes = ((size_t)1 << log_n) * sizeof(fe);
  fe* d = nullptr;
  ZK_TRY("zk::dmalloc(ntt data)", zk::dmalloc((void**)&d, bytes, s));
  cudaError_t e = zk::h2d_copy(d, a, bytes, s);
  if (e == cudaSuccess) {
    st = ntt_device(device, d, log_n, load_fr(omega), coset, post, s);
    if (st == ZKGPU_OK) e = zk::d2h_copy(a, d, bytes, s);
  }
  cudaFreeAsync(d, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (st) return st;
  if (e != cudaSuccess) return zk::status_of("ntt_host copy", e);
  return zk::status_of("ntt_host sync", e2);
}

// LDE pipeline on device buffers.
int lde_device(int device, const fe* d_values, uint32_t log_n, fe* d_ext, uint32_t log_ext, const hf::Fr& w_inv,
               const hf::Fr& divisor, const hf::Fr& g, const hf::Fr& w_ext, cudaStream_t s) {
  const size_t n = (size_t)1 << log_n, N = (size_t)1 << log_ext;
  if (log_n < 3) {
    // tiny domains: coefficients in the first n slots, zero tail, two transforms
    ZK_TRY("lde copy", cudaMemcpyAsync(d_ext, d_values, n * sizeof(fe), cudaMemcpyDeviceToDevice, s));
    if (N > n) ZK_TRY("lde zero", cudaMemsetAsync(d_ext + n, 0, (N - n) * sizeof(fe), s));
    int st = ntt_device(device, d_ext, log_n, w_inv, nullptr, &divisor, s);
    if (st) return st;
    return ntt_device(device, d_ext, log_ext, w_ext, &g, nullptr, s);
  }
  // 1) ifft of the values, read in place from d_values, written to d_ext[0, n);
  //    its last pass multiplies output i by n^-1 * g^i (the coset shift)
  // 2) NTT of d_ext on the extended domain; its first pass treats the zero
  //    padding [n, N) as known zeros, so the tail is never written or read
  cudaError_t e;
  const zk::NttTablesRef ti = zk::ntt_tables_get(device, w_inv, (int)log_n, s, &e);
  if (!ti) return zk::status_of("ntt_tables_get", e);
  const zk::NttTablesRef te = zk::ntt_tables_get(device, w_ext, (int)log_ext, s, &e);
  if (!te) return zk::status_of("ntt_tables_get", e);
  const zk::PowTablesRef gd = zk::pow_tables_get(device, g, (int)log_n, s, &e, &divisor);
  if (!gd) return zk::status_of("pow_tables_get", e);
  fe* tmp = nullptr;
  ZK_TRY("zk::dmalloc(lde scratch)", zk::dmalloc((void**)&tmp, N * sizeof(fe), s));
  // the skip works on whole rows of the first pass; otherwise zero the tail
  if (te->plan.npass > 1 && N > n && n % (1ull << (log_ext - te->plan.bits[0])) != 0)
    ZK_TRY("lde zero", cudaMemsetAsync(d_ext + n, 0, (N - n) * sizeof(fe), s));
  zk::NttFuse f1;
  f1.src = d_values;
  f1.post_tab = gd.get();
  e = zk::ntt_run(*ti, d_ext, tmp, f1, s);
  zk::count_launches(ti->plan.npass);
  if (e == cudaSuccess) {
    zk::NttFuse f2;
    f2.nonzero = n;
    e = zk::ntt_run(*te, d_ext, tmp, f2, s);
    zk::count_launches(te->plan.npass);
  }
  cudaFreeAsync(tmp, s);
  return zk::status_of("lde", e);
}

// Extended -> coefficient form (the inverse of the LDE): ifft over the
// extended domain, times N^-1 * g_inv^i, first m coefficients to d_out.
// The scale and the coset powers ride on the ifft's last pass (one table).
int ext_to_coeff_device(int device, const fe* d_ext, uint32_t log_ext, const hf::Fr& w_inv, const hf::Fr& divisor,
                        const hf::Fr& g_inv, fe* d_out, uint64_t m, cudaStream_t s) {
  const size_t N = (size_t)1 << log_ext;
  cudaError_t e;
  const zk::NttTablesRef t = zk::ntt_tables_get(device, w_inv, (int)log_ext, s, &e);
  if (!t) return zk::status_of("ntt_tables_get", e);
  const bool tiny = t->plan.npass == 0;  // direct kernel: constant scale only
  const zk::PowTablesRef gd = zk::pow_tables_get(device, g_inv, (int)log_ext, s, &e, tiny ? nullptr : &divisor);
  if (!gd) return zk::status_of("pow_tables_get", e);
  fe *work = nullptr, *tmp = nullptr;
  ZK_TRY("zk::dmalloc(ext_to_coeff work)", zk::dmalloc((void**)&work, N * sizeof(fe), s));
  if (t->plan.npass > 1) {
    e = zk::dmalloc((void**)&tmp, N * sizeof(fe), s);
    if (e != cudaSuccess) {
      cudaFreeAsync(work, s);
      return zk::status_of("zk::dmalloc(ext_to_coeff scratch)", e);
    }
  }
  if (tiny) {
    e = cudaMemcpyAsync(work, d_ext, N * sizeof(fe), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = zk::ntt_run(*t, work, tmp, nullptr, &divisor, s);
    if (e == cudaSuccess) e = zk::fr_scale_copy(d_out, work, m, 1, gd.get(), s);
    zk::count_launches(2);
  } else {
    zk::NttFuse f;
    f.src = d_ext;
    f.post_tab = gd.get();
    e = zk::ntt_run(*t, work, tmp, f, s);
    zk::count_launches(t->plan.npass);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, work, m * sizeof(fe), cudaMemcpyDeviceToDevice, s);
  }
  cudaFreeAsync(work, s);
  if (tmp) cudaFreeAsync(tmp, s);
  return zk::status_of("ext_to_coeff", e);
}

int check_etc_args(uint32_t log_ext, const uint64_t* omega_ext_inv, const uint64_t* divisor, const uint64_t* g_inv,
                   uint64_t m) {
  if (!omega_ext_inv || !divisor || !g_inv) return ZKGPU_EINVAL;
  if (log_ext > (uint32_t)zk::NTT_MAX_LOG || m > (1ull << log_ext)) return ZKGPU_EINVAL;
  hf::Fr w = load_fr(omega_ext_inv), d = load_fr(divisor), g = load_fr(g_inv);
  if (!hf::is_canonical(w) || !hf::is_canonical(d) || !hf::is_canonical(g)) return ZKGPU_EINVAL;
  if (!hf::is_primitive_root(w, log_ext)) return ZKGPU_EINVAL;
  return ZKGPU_OK;
}

}  // namespace

// ===========================================================================
// reference-compatible symbols (src/api.rs:3-14)
// ===========================================================================
extern "C" uint64_t parallel_fft_api(size_t device_id, uint64_t* req, const uint64_t* omega, const uint64_t* twiddle,
                                     uint64_t n, uint64_t log_n, uint64_t twiddle_size) {
  (void)twiddle;
  (void)twiddle_size;
  if (log_n > 63 || n != (1ull << log_n)) return ZKGPU_EINVAL;
  return (uint64_t)ntt_host((int)device_id, req, (uint32_t)log_n, omega, nullptr, nullptr);
}

extern "C" uint64_t parallel_ifft_api(size_t device_id, uint64_t* req, const uint64_t* omega, const uint64_t* twiddle,
                                      uint64_t n, uint64_t log_n, uint64_t twiddle_size, const uint64_t* divisor) {
  (void)twiddle;
  (void)twiddle_size;
  if (log_n > 63 || n != (1ull << log_n) || !divisor) return ZKGPU_EINVAL;
  hf::Fr d = load_fr(divisor);
  if (!hf::is_canonical(d)) return ZKGPU_EINVAL;
  return (uint64_t)ntt_host((int)device_id, req, (uint32_t)log_n, omega, nullptr, &d);
}

extern "C" uint64_t parallel_coeff_to_extended_part_api(size_t device_id, uint64_t* req, const uint64_t* omega,
                                                        const uint64_t* twiddle, uint64_t n, uint64_t log_n,
                                                        uint64_t twiddle_size, const uint64_t* c) {
  (void)twiddle;
  (void)twiddle_size;
  if (log_n > 63 || n != (1ull << log_n) || !c) return ZKGPU_EINVAL;
  hf::Fr cc = load_fr(c);
  if (!hf::is_canonical(cc)) return ZKGPU_EINVAL;
  return (uint64_t)ntt_host((int)device_id, req, (uint32_t)log_n, omega, &cc, nullptr);
}

// ===========================================================================
// short names (fft / ifft / coset_fft / msm), host buffers
// ===========================================================================
extern "C" int zkgpu_fft(int device, uint64_t* a, uint32_t log_n, const uint64_t omega[4]) {
  return ntt_host(device, a, log_n, omega, nullptr, nullptr);
}

extern "C" int zkgpu_ifft(int device, uint64_t* a, uint32_t log_n, const uint64_t omega_inv[4],
                          const uint64_t divisor[4]) {
  if (!divisor) return ZKGPU_EINVAL;
  hf::Fr d = load_fr(divisor);
  if (!hf::is_canonical(d)) return ZKGPU_EINVAL;
  return ntt_host(device, a, log_n, omega_inv, nullptr, &d);
}

extern "C" int zkgpu_coset_fft(int device, uint64_t* a, uint32_t log_n, const uint64_t omega[4], const uint64_t c[4]) {
  if (!c) return ZKGPU_EINVAL;
  hf::Fr cc = load_fr(c);
  if (!hf::is_canonical(cc)) return ZKGPU_EINVAL;
  return ntt_host(device, a, log_n, omega, &cc, nullptr);
}

static int check_lde_args(uint32_t log_n, uint32_t log_ext, const uint64_t* omega_inv, const uint64_t* divisor,
                          const uint64_t* g, const uint64_t* omega_ext) {
  if (!omega_inv || !divisor || !g || !omega_ext) return ZKGPU_EINVAL;
  if (log_ext < log_n || log_ext > (uint32_t)zk::NTT_MAX_LOG) return ZKGPU_EINVAL;
  hf::Fr wi = load_fr(omega_inv), d = load_fr(divisor), gg = load_fr(g), we = load_fr(omega_ext);
  if (!hf::is_canonical(wi) || !hf::is_canonical(d) || !hf::is_canonical(gg) || !hf::is_canonical(we))
    return ZKGPU_EINVAL;
  if (!hf::is_primitive_root(wi, log_n) || !hf::is_primitive_root(we, log_ext)) return ZKGPU_EINVAL;
  return ZKGPU_OK;
}

extern "C" int zkgpu_lagrange_to_extended(int device, const uint64_t* values, uint32_t log_n, uint64_t* ext,
                                          uint32_t log_ext, const uint64_t omega_inv[4], const uint64_t divisor[4],
                                          const uint64_t g[4], const uint64_t omega_ext[4]) {
  if (!values || !ext) return ZKGPU_EINVAL;
  int st = check_lde_args(log_n, log_ext, omega_inv, divisor, g, omega_ext);
  if (st) return st;
  cudaStream_t s;
  st = zk::bind_device(device, &s);
  if (st) return st;
  const size_t n = (size_t)1 << log_n, N = (size_t)1 << log_ext;
  fe *d_in = nullptr, *d_ext = nullptr;
  ZK_TRY("zk::dmalloc(lde in)", zk::dmalloc((void**)&d_in, n * sizeof(fe), s));
  cudaError_t e = zk::dmalloc((void**)&d_ext, N * sizeof(fe), s);
  if (e != cudaSuccess) {
    cudaFreeAsync(d_in, s);
    return zk::status_of("zk::dmalloc(lde ext)", e);
  }
  e = zk::h2d_copy(d_in, values, n * sizeof(fe), s);
  if (e == cudaSuccess) {
    st = lde_device(device, d_in, log_n, d_ext, log_ext, load_fr(omega_inv), load_fr(divisor), load_fr(g),
                    load_fr(omega_ext), s);
    if (st == ZKGPU_OK) e = zk::d2h_copy(ext, d_ext, N * sizeof(fe), s);
  }
  cudaFreeAsync(d_in, s);
  cudaFreeAsync(d_ext, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (st) return st;
  if (e != cudaSuccess) return zk::status_of("lde copy", e);
  return zk::status_of("lde sync", e2);
}

// ===========================================================================
// device-resident API
// ===========================================================================
extern "C" int zkgpu_ntt_dev(int device, uint64_t* d_a, uint32_t log_n, const uint64_t omega[4],
                             const uint64_t* coset_c, const uint64_t* post_scale, void* stream) {
  int st = check_ntt_args(d_a, omega, log_n);
  if (st) return st;
  hf::Fr c, ps;
  if (coset_c) {
    c = load_fr(coset_c);
    if (!hf::is_canonical(c)) return ZKGPU_EINVAL;
  }
  if (post_scale) {
    ps = load_fr(post_scale);
    if (!hf::is_canonical(ps)) return ZKGPU_EINVAL;
  }
  cudaStream_t own;
  st = zk::bind_device(device, &own);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  return ntt_device(device, reinterpret_cast<fe*>(d_a), log_n, load_fr(omega), coset_c ? &c : nullptr,
                    post_scale ? &ps : nullptr, s);
}

extern "C" int zkgpu_lagrange_to_extended_dev(int device, const uint64_t* d_values, uint32_t log_n, uint64_t* d_ext,
                                              uint32_t log_ext, const uint64_t omega_inv[4], const uint64_t divisor[4],
                                              const uint64_t g[4], const uint64_t omega_ext[4], void* stream) {
  if (!d_values || !d_ext) return ZKGPU_EINVAL;
  int st = check_lde_args(log_n, log_ext, omega_inv, divisor, g, omega_ext);
  if (st) return st;
  cudaStream_t own;
  st = zk::bind_device(device, &own);
  if (st) return st;
  return lde_device(device, reinterpret_cast<const fe*>(d_values), log_n, reinterpret_cast<fe*>(d_ext), log_ext,
                    load_fr(omega_inv), load_fr(divisor), load_fr(g), load_fr(omega_ext), (cudaStream_t)stream);
}

extern "C" int zkgpu_extended_to_coeff(int device, const uint64_t* ext, uint32_t log_ext, uint64_t* out, uint64_t m,
                                       const uint64_t omega_ext_inv[4], const uint64_t ext_divisor[4],
                                       const uint64_t g_inv[4]) {
  if (!ext || (m && !out)) return ZKGPU_EINVAL;
  int st = check_etc_args(log_ext, omega_ext_inv, ext_divisor, g_inv, m);
  if (st) return st;
  if (m == 0) return ZKGPU_OK;
  cudaStream_t s;
  st = zk::bind_device(device, &s);
  if (st) return st;
  const size_t N = (size_t)1 << log_ext;
  fe *d_ext = nullptr, *d_out = nullptr;
  ZK_TRY("zk::dmalloc(ext_to_coeff in)", zk::dmalloc((void**)&d_ext, N * sizeof(fe), s));
  cudaError_t e = zk::dmalloc((void**)&d_out, m * sizeof(fe), s);
  if (e != cudaSuccess) {
    cudaFreeAsync(d_ext, s);
    return zk::status_of("zk::dmalloc(ext_to_coeff out)", e);
  }
  e = zk::h2d_copy(d_ext, ext, N * sizeof(fe), s);
  if (e == cudaSuccess) {
    st = ext_to_coeff_device(device, d_ext, log_ext, load_fr(omega_ext_inv), load_fr(ext_divisor), load_fr(g_inv),
                             d_out, m, s);
    if (st == ZKGPU_OK) e = zk::d2h_copy(out, d_out, m * sizeof(fe), s);
  }
  cudaFreeAsync(d_ext, s);
  cudaFreeAsync(d_out, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (st) return st;
  if (e != cudaSuccess) return zk::status_of("ext_to_coeff copy", e);
  return zk::status_of("ext_to_coeff sync", e2);
}

extern "C" int zkgpu_extended_to_coeff_dev(int device, const uint64_t* d_ext, uint32_t log_ext, uint64_t* d_out,
                                           uint64_t m, const uint64_t omega_ext_inv[4], const uint64_t ext_divisor[4],
                                           const uint64_t g_inv[4], void* stream) {
  if (!d_ext || (m && !d_out)) return ZKGPU_EINVAL;
  int st = check_etc_args(log_ext, omega_ext_inv, ext_divisor, g_inv, m);
  if (st) return st;
  if (m == 0) return ZKGPU_OK;
  cudaStream_t own;
  st = zk::bind_device(device, &own);
  if (st) return st;
  return ext_to_coeff_device(device, reinterpret_cast<const fe*>(d_ext), log_ext, load_fr(omega_ext_inv),
                             load_fr(ext_divisor), load_fr(g_inv), reinterpret_cast<fe*>(d_out), m,
                             (cudaStream_t)stream);
}

// ===========================================================================
// diagnostics
// ===========================================================================
namespace {
template <class P>
__global__ void field_op_kernel(int op, const fe* a, const fe* b, fe* out, uint64_t n) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t x[8], y[8], r[8];
  zk::ld_fe(x, a + i);
  zk::ld_fe(y, b + i);
  if (op == 0)
    zk::mul<P>(r, x, y);
  else if (op == 1)
    zk::add<P>(r, x, y);
  else if (op == 2)
    zk::sub<P>(r, x, y);
  else
    zk::fq_inv_divsteps(r, x);  // op 3, Fq only (checked on the host): the MSM rounds' inversion
  zk::st_fe(out + i, r);
}
}  // namespace

extern "C" int zkgpu_field_op(int device, int op, int fid, const uint64_t* a, const uint64_t* b, uint64_t* out,
                              uint64_t n) {
  if (!a || (op != 3 && !b) || !out || op < 0 || op > 3 || fid < 0 || fid > 1 || (op == 3 && fid != 1))
    return ZKGPU_EINVAL;
  if (op == 3) b = a;  // unused operand
  if (n == 0) return ZKGPU_OK;
  cudaStream_t s;
  int st = zk::bind_device(device, &s);
  if (st) return st;
  const size_t bytes = n * sizeof(fe);
  fe *da = nullptr, *db = nullptr, *dout = nullptr;
  ZK_TRY("cudaMallocAsync", zk::dmalloc((void**)&da, bytes, s));
  ZK_TRY("cudaMallocAsync", zk::dmalloc((void**)&db, bytes, s));
  ZK_TRY("cudaMallocAsync", zk::dmalloc((void**)&dout, bytes, s));
  zk::h2d_copy(da, a, bytes, s);
  zk::h2d_copy(db, b, bytes, s);
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (fid == 0)
    field_op_kernel<zk::FrP><<<grid, 256, 0, s>>>(op, da, db, dout, n);
  else
    field_op_kernel<zk::FqP><<<grid, 256, 0, s>>>(op, da, db, dout, n);
  zk::count_launches(1);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = zk::d2h_copy(out, dout, bytes, s);
  cudaFreeAsync(da, s);
  cudaFreeAsync(db, s);
  cudaFreeAsync(dout, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return zk::status_of("field_op", e);
  return zk::status_of("field_op sync", e2);
}

// cuda/fft.cu:554-558 ran a throw-away kernel; here: a device known-answer
// check of the Fr and Fq products against the host arithmetic.
extern "C" uint64_t do_fft_ffi(size_t device_id) {
  uint64_t a[2][4] = {{0x1234567890abcdefULL, 0x0fedcba987654321ULL, 0x1111111111111111ULL, 0x0222222222222222ULL},
                      {0x9191727205810674ULL, 0x8873516619432482ULL, 0x6234034562745979ULL, 0x1723971208416369ULL}};
  uint64_t b[2][4] = {{0x9191727205810674ULL, 0x8873516619432482ULL, 0x6234034562745979ULL, 0x1723971208416369ULL},
                      {0x1234567890abcdefULL, 0x0fedcba987654321ULL, 0x1111111111111111ULL, 0x0222222222222222ULL}};
  uint64_t out[2][4];
  int st = zkgpu_field_op((int)device_id, 0, 0, &a[0][0], &b[0][0], &out[0][0], 2);
  if (st) return (uint64_t)st;
  for (int i = 0; i < 2; i++) {
    hf::Fr x, y;
    std::memcpy(x.v, a[i], 32);
    std::memcpy(y.v, b[i], 32);
    hf::Fr r = hf::mul(x, y);
    if (std::memcmp(r.v, out[i], 32) != 0) return ZKGPU_ECUDA;
  }
  return ZKGPU_OK;
}
