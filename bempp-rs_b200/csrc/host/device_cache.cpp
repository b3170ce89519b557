// Process-wide cache of device memory blocks for DeviceBuffer (see core.h).
//
// Blocks are rounded up (to 64 KiB below 2 MiB, to 2 MiB above) and kept per device in a
// free list ordered by size; a request takes the smallest free block of its device that
// is at least as large and at most twice as large.  Free blocks beyond kCacheBytes per
// device are released, largest first.  When cudaMalloc fails, the device's free blocks are
// released and the allocation is tried once more.
#include <map>
#include <mutex>

#include "core.h"

namespace bempp_b200 {
namespace {

constexpr size_t kCacheBytes = size_t(4) << 30;

struct Block {
  int device;
  size_t size;
};

struct Cache {
  std::mutex mu;
  std::map<void*, Block> used;
  std::map<int, std::multimap<size_t, void*>> free;  // device -> size -> block
  std::map<int, size_t> free_bytes;
};

// Never destroyed: DeviceBuffers owned by other static objects return their blocks while
// the process exits, after this file's own statics would have been destroyed.
Cache& cache() {
  static Cache* c = new Cache;
  return *c;
}

size_t rounded(size_t n) {
  const size_t g = n < (size_t(2) << 20) ? (size_t(64) << 10) : (size_t(2) << 20);
  return (n + g - 1) / g * g;
}

// Releases free blocks of `device` until at most `keep` bytes remain (mu held).
size_t release(Cache& c, int device, size_t keep) {
  auto& fl = c.free[device];
  size_t released = 0;
  while (c.free_bytes[device] > keep && !fl.empty()) {
    auto big = std::prev(fl.end());
    cudaFree(big->second);
    c.free_bytes[device] -= big->first;
    released += big->first;
    fl.erase(big);
  }
  return released;
}

}  // namespace

cudaError_t device_cache_alloc(void** ptr, size_t bytes) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  const size_t size = rounded(bytes);
  Cache& c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  auto& fl = c.free[device];
  auto it = fl.lower_bound(size);
  if (it != fl.end() && it->first <= 2 * size) {
    *ptr = it->second;
    c.used[*ptr] = Block{device, it->first};
    c.free_bytes[device] -= it->first;
    fl.erase(it);
    return cudaSuccess;
  }
  e = cudaMalloc(ptr, size);
  if (e == cudaErrorMemoryAllocation && c.free_bytes[device] > 0) {
    cudaGetLastError();  // clear the allocation error before retrying
    release(c, device, 0);
    e = cudaMalloc(ptr, size);
  }
  if (e != cudaSuccess) return e;
  c.used[*ptr] = Block{device, size};
  return cudaSuccess;
}

void device_cache_free(void* ptr) {
  if (!ptr) return;
  Cache& c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  auto it = c.used.find(ptr);
  if (it == c.used.end()) return;
  const Block b = it->second;
  c.used.erase(it);
  // the block may still be read or written by work in flight (on any stream): wait for
  // the device, as cudaFree would, before another request can take it
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != b.device) cudaSetDevice(b.device);
  cudaDeviceSynchronize();
  if (cur != b.device) cudaSetDevice(cur);
  c.free[b.device].emplace(b.size, ptr);
  c.free_bytes[b.device] += b.size;
  release(c, b.device, kCacheBytes);
}

size_t device_cache_trim() {
  Cache& c = cache();
  std::lock_guard<std::mutex> lock(c.mu);
  size_t released = 0;
  for (auto& d : c.free) released += release(c, d.first, 0);
  return released;
}

}  // namespace bempp_b200
