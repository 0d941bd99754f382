// table_cache.cu — the per-device caches of NTT root / twist tables and of
// coset power tables (declared in ntt.cuh).
//
// A table is built on the first call that needs it and shared by every later
// one: the reference rebuilt and re-uploaded its twiddle table on every call
// (cuda/fft.cu:282-285).  Entries are reference-counted: the cache holds one
// reference, and work that reads a table (an enqueued transform, a batch
// graph, a serving wave) holds another until it is done.  The cache is capped
// per device (ZKGPU_TABLE_CACHE_MB, default 8192 MiB) and evicts its least
// recently used entries when a new one would exceed the cap; an evicted table
// is freed (cudaFree, which waits for the device) when its last holder lets
// go.  Tables are built outside the cache lock, so a first use on one thread
// does not stall lookups on others.
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "ntt.cuh"
#include "runtime.cuh"

namespace zk {

namespace {

struct NttKey {
  int dev;
  int log_n;
  uint64_t w[4];
  uint32_t plan;  // pass widths, 6 bits each
  bool operator<(const NttKey& o) const {
    return std::tie(dev, log_n, w[0], w[1], w[2], w[3], plan) <
           std::tie(o.dev, o.log_n, o.w[0], o.w[1], o.w[2], o.w[3], o.plan);
  }
};
struct PowKey {
  int dev, log_n;
  uint64_t c[4], s[4];
  bool operator<(const PowKey& o) const {
    return std::tie(dev, log_n, c[0], c[1], c[2], c[3], s[0], s[1], s[2], s[3]) <
           std::tie(o.dev, o.log_n, o.c[0], o.c[1], o.c[2], o.c[3], o.s[0], o.s[1], o.s[2], o.s[3]);
  }
};
template <class T>
struct Entry {
  std::shared_ptr<const T> ref;
  uint64_t bytes = 0;
  uint64_t last_use = 0;
};

std::mutex g_mu;
std::map<NttKey, Entry<NttTables>> g_ntt;
std::map<PowKey, Entry<PowTables>> g_pow;
std::map<int, uint64_t> g_bytes;  // per device
std::map<int, uint64_t> g_builds;  // tables built (misses), per device
uint64_t g_tick = 0;

uint64_t cap_bytes() {
  static const uint64_t cap = [] {
    const char* v = std::getenv("ZKGPU_TABLE_CACHE_MB");
    const uint64_t mb = v && *v ? std::strtoull(v, nullptr, 10) : 8192ull;
    return mb << 20;
  }();
  return cap;
}

uint32_t plan_code(const NttPlan& p) {
  uint32_t c = (uint32_t)p.npass;
  for (int k = 0; k < NTT_MAX_PASS; k++) c = (c << 6) | (uint32_t)p.bits[k];
  return c;
}

// with g_mu held: drop least recently used entries of `dev` until `extra`
// more bytes fit under the cap; the dropped references go to `drop` so that
// any frees they trigger happen after the lock is released
template <class V>
void evict_for(int dev, uint64_t extra, V& drop) {
  for (;;) {
    if (g_bytes[dev] + extra <= cap_bytes()) return;
    uint64_t oldest = ~0ull;
    int which = -1;
    auto n_old = g_ntt.end();
    auto p_old = g_pow.end();
    for (auto it = g_ntt.begin(); it != g_ntt.end(); ++it)
      if (it->first.dev == dev && it->second.last_use < oldest) {
        oldest = it->second.last_use;
        n_old = it;
        which = 0;
      }
    for (auto it = g_pow.begin(); it != g_pow.end(); ++it)
      if (it->first.dev == dev && it->second.last_use < oldest) {
        oldest = it->second.last_use;
        p_old = it;
        which = 1;
      }
    if (which < 0) return;  // nothing left to evict: the new entry alone exceeds the cap
    if (which == 0) {
      g_bytes[dev] -= n_old->second.bytes;
      drop.push_back(n_old->second.ref);
      g_ntt.erase(n_old);
    } else {
      g_bytes[dev] -= p_old->second.bytes;
      drop.push_back(p_old->second.ref);
      g_pow.erase(p_old);
    }
  }
}

void free_ntt(const NttTables* t) {
  NttTables* m = const_cast<NttTables*>(t);
  ntt_tables_release(m);
  delete m;
}
void free_pow(const PowTables* t) {
  if (t->lo) cudaFree(t->lo);
  if (t->hi) cudaFree(t->hi);
  delete t;
}

}  // namespace

NttTablesRef ntt_tables_get(int device, const host::Fr& omega, int log_n, cudaStream_t s, cudaError_t* err) {
  // the plan is the autotuner's choice for this device and size, if any;
  // tables of an older choice stay alive while work still holds them
  const NttPlan plan = tuned_ntt_plan(device, log_n);
  const NttKey key{device, log_n, {omega.v[0], omega.v[1], omega.v[2], omega.v[3]}, plan_code(plan)};
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_ntt.find(key);
    if (it != g_ntt.end()) {
      it->second.last_use = ++g_tick;
      *err = cudaSuccess;
      return it->second.ref;
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_builds[device]++;
  }
  NttTables* t = new NttTables();
  cudaError_t e = ntt_tables_build(t, plan, omega, s);  // synchronises s
  if (e != cudaSuccess) {
    delete t;
    *err = e;
    return nullptr;
  }
  NttTablesRef ref(t, free_ntt);
  std::vector<std::shared_ptr<const void>> drop;
  NttTablesRef out;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_ntt.find(key);
    if (it != g_ntt.end()) {  // another thread built the same tables meanwhile: use theirs
      it->second.last_use = ++g_tick;
      out = it->second.ref;
    } else {
      evict_for(device, t->bytes, drop);
      g_ntt[key] = Entry<NttTables>{ref, t->bytes, ++g_tick};
      g_bytes[device] += t->bytes;
      out = ref;
    }
  }
  *err = cudaSuccess;
  return out;
}

PowTablesRef pow_tables_get(int device, const host::Fr& c, int log_n, cudaStream_t s, cudaError_t* err,
                            const host::Fr* scale) {
  const host::Fr one = host::one();
  const host::Fr& sc = scale ? *scale : one;
  const PowKey key{device, log_n, {c.v[0], c.v[1], c.v[2], c.v[3]}, {sc.v[0], sc.v[1], sc.v[2], sc.v[3]}};
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_pow.find(key);
    if (it != g_pow.end()) {
      it->second.last_use = ++g_tick;
      *err = cudaSuccess;
      return it->second.ref;
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_builds[device]++;
  }
  PowTables* t = new PowTables();
  cudaError_t e = pow_tables_make(t, c, log_n, s, scale, false);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    if (t->lo) cudaFree(t->lo);
    if (t->hi) cudaFree(t->hi);
    delete t;
    *err = e;
    return nullptr;
  }
  const uint64_t bytes = ((1ull << t->shift) + (1ull << (log_n > (int)t->shift ? log_n - t->shift : 0))) * sizeof(fe);
  PowTablesRef ref(t, free_pow);
  std::vector<std::shared_ptr<const void>> drop;
  PowTablesRef out;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_pow.find(key);
    if (it != g_pow.end()) {
      it->second.last_use = ++g_tick;
      out = it->second.ref;
    } else {
      evict_for(device, bytes, drop);
      g_pow[key] = Entry<PowTables>{ref, bytes, ++g_tick};
      g_bytes[device] += bytes;
      out = ref;
    }
  }
  *err = cudaSuccess;
  return out;
}

uint64_t table_cache_builds(int device) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_builds.find(device);
  return it == g_builds.end() ? 0 : it->second;
}

uint64_t table_cache_bytes(int device) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_bytes.find(device);
  return it == g_bytes.end() ? 0 : it->second;
}

void table_cache_clear(int device) {
  std::vector<std::shared_ptr<const void>> drop;  // released after the lock (cudaFree waits for the device)
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto it = g_ntt.begin(); it != g_ntt.end();) {
    if (it->first.dev == device) {
      drop.push_back(it->second.ref);
      it = g_ntt.erase(it);
    } else {
      ++it;
    }
  }
  for (auto it = g_pow.begin(); it != g_pow.end();) {
    if (it->first.dev == device) {
      drop.push_back(it->second.ref);
      it = g_pow.erase(it);
    } else {
      ++it;
    }
  }
  g_bytes[device] = 0;
}

}  // namespace zk

extern "C" int zkgpu_release_cached(int device) {
  cudaStream_t s;
  int st = zk::bind_device(device, &s);
  if (st) return st;
  zk::table_cache_clear(device);
  return zk::status_of("zkgpu_release_cached", zk::trim_pool(device));
}
