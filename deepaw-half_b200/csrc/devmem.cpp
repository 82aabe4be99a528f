// Caching device allocator (see devmem.h).
#include "devmem.h"

#include <atomic>

#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include "common.h"

namespace hb {

namespace {

using Key = std::pair<int, size_t>;   // (device, bytes)
using Pool = std::multimap<Key, void*>;

constexpr size_t kThreadCap = size_t(16) << 30;   // cached bytes kept per thread

size_t round_bytes(size_t b) {
  if (b <= (size_t(1) << 20)) return (b + 511) & ~size_t(511);
  return (b + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
}

void timed_free(void* p, size_t bytes) {
  AllocTimer timer("cudaFree", bytes);
  cudaFree(p);
}

std::mutex g_mu;
Pool g_pool;

// Smallest block in [key.bytes, 2 key.bytes] on the same device, removed from pool.
void* take(Pool& pool, const Key& key, size_t* granted) {
  auto it = pool.lower_bound(key);
  if (it == pool.end() || it->first.first != key.first || it->first.second > 2 * key.second) return nullptr;
  void* p = it->second;
  *granted = it->first.second;
  pool.erase(it);
  return p;
}

struct ThreadCache {
  Pool pool;
  size_t bytes = 0;
  ~ThreadCache() {
    if (pool.empty()) return;
    cudaDeviceSynchronize();   // every use of these blocks has finished
    std::lock_guard<std::mutex> lock(g_mu);
    for (auto& kv : pool) g_pool.insert(kv);
    pool.clear();
  }
};

thread_local ThreadCache t_cache;
std::atomic<long long> g_requests{0}, g_driver_allocs{0};

void release_all_locked() {
  for (auto& kv : g_pool) timed_free(kv.second, kv.first.second);
  g_pool.clear();
}

}  // namespace

void* device_alloc(size_t bytes, size_t* granted) {
  g_requests.fetch_add(1, std::memory_order_relaxed);
  int dev = 0;
  cudaGetDevice(&dev);
  const Key key{dev, round_bytes(bytes)};
  if (void* p = take(t_cache.pool, key, granted)) {
    t_cache.bytes -= *granted;
    return p;
  }
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (void* p = take(g_pool, key, granted)) return p;
  }
  void* p = nullptr;
  cudaError_t e;
  {
    AllocTimer timer("cudaMalloc", key.second);
    g_driver_allocs.fetch_add(1, std::memory_order_relaxed);
    e = cudaMalloc(&p, key.second);
  }
  if (e != cudaSuccess) {   // give the cache back and retry once
    cudaGetLastError();
    device_cache_release();
    AllocTimer timer("cudaMalloc", key.second);
    g_driver_allocs.fetch_add(1, std::memory_order_relaxed);
    e = cudaMalloc(&p, key.second);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(kInternal, "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  *granted = key.second;
  return p;
}

void device_free(void* p, size_t granted) {
  if (!p) return;
  if (t_cache.bytes + granted > kThreadCap) {
    timed_free(p, granted);
    return;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  t_cache.pool.insert({Key{dev, granted}, p});
  t_cache.bytes += granted;
}

void device_alloc_counts(long long* requests, long long* driver_allocations) {
  if (requests) *requests = g_requests.load(std::memory_order_relaxed);
  if (driver_allocations) *driver_allocations = g_driver_allocs.load(std::memory_order_relaxed);
}

void device_cache_release() {
  cudaDeviceSynchronize();
  for (auto& kv : t_cache.pool) timed_free(kv.second, kv.first.second);
  t_cache.pool.clear();
  t_cache.bytes = 0;
  std::lock_guard<std::mutex> lock(g_mu);
  release_all_locked();
}

}  // namespace hb
