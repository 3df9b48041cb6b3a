// Page-locked host blocks for callers that keep their spin buffers on the
// host (the cxxjij systems): a copy between page-locked memory and the device
// is one DMA at the link's rate, with no staging through the driver's bounce
// buffers, and it overlaps other work on the stream.
//
// Page-locking is slow (the pages are faulted in and pinned) and page-locked
// memory is scarce, so freed blocks stay in a process-wide cache and serve the
// next request of at most their size and at least half of it; the cache keeps
// at most kCacheBytes and returns the largest blocks to the system past that.
// Blocks are page-locked through the device of the last context created in
// the process (a block is usable from every context), so that a request made
// before any context exists creates none on some default device: such a block
// is ordinary memory.  So is every block when page-locked memory cannot be had
// (no device, or the system refuses) or OJ_HOST_PINNED=0 is in the
// environment; every entry point accepts ordinary memory as well.  The cache is never torn down: its
// blocks go back to the system with the process (a cudaFreeHost from a static
// destructor could run after the CUDA runtime is gone).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <iterator>
#include <map>
#include <mutex>
#include <unordered_map>

#include "oj_internal.h"
#include "openjij_b200.h"

namespace {

constexpr size_t kCacheBytes = size_t(2) << 30;
constexpr size_t kGrain = size_t(64) << 10;  // blocks are whole multiples of this

struct HostCache {
  std::mutex mu;
  std::multimap<size_t, void*> free_blocks;      // size -> block
  std::unordered_map<void*, size_t> pinned_size;  // every page-locked block handed out or cached
  size_t cached = 0;
};

HostCache& cache() {
  static HostCache* c = new HostCache();  // never destroyed
  return *c;
}

std::atomic<int> g_pin_device{-1};

bool pinning_enabled() {
  const char* env = std::getenv("OJ_HOST_PINNED");
  return !(env && env[0] == '0');
}

}  // namespace

namespace oj {
void host_pin_device(int device) { g_pin_device.store(device); }
}  // namespace oj

extern "C" void* oj_host_alloc(size_t bytes) {
  const size_t want = bytes == 0 ? kGrain : (bytes + kGrain - 1) / kGrain * kGrain;
  const int dev = g_pin_device.load();
  if (dev >= 0 && pinning_enabled()) {
    HostCache& c = cache();
    {
      std::lock_guard<std::mutex> lk(c.mu);
      auto it = c.free_blocks.lower_bound(want);
      if (it != c.free_blocks.end() && it->first <= 2 * want) {
        void* p = it->second;
        c.cached -= it->first;
        c.free_blocks.erase(it);
        return p;
      }
    }
    void* p = nullptr;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
    const cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocPortable);
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    if (e == cudaSuccess && p) {
      std::lock_guard<std::mutex> lk(c.mu);
      c.pinned_size[p] = want;
      return p;
    }
    cudaGetLastError();  // no device or no page-locked memory: ordinary memory below
  }
  return std::malloc(want);
}

extern "C" void oj_host_free(void* p) {
  if (!p) return;
  HostCache& c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  const auto it = c.pinned_size.find(p);
  if (it == c.pinned_size.end()) {
    std::free(p);
    return;
  }
  c.free_blocks.emplace(it->second, p);
  c.cached += it->second;
  while (c.cached > kCacheBytes && !c.free_blocks.empty()) {
    auto big = std::prev(c.free_blocks.end());
    c.cached -= big->first;
    c.pinned_size.erase(big->second);
    cudaFreeHost(big->second);
    c.free_blocks.erase(big);
  }
}

extern "C" int32_t oj_host_is_pinned(const void* p) {
  HostCache& c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  return c.pinned_size.count(const_cast<void*>(p)) ? 1 : 0;
}
