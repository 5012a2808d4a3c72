// Caching allocators for device and pinned host blocks.
//
// cudaMalloc / cudaFree (and cudaMallocHost / cudaFreeHost) take device-wide
// locks, synchronise and cost milliseconds each; a solve handle holds some
// forty buffers, so creating and destroying handles (one per served request,
// one per end-to-end call) spent more time allocating than solving. Freed
// blocks are kept here, per device and per rounded size, and handed to the
// next allocation of the same size class. A block is only returned by an
// owner whose stream has drained, so a reused block has no work in flight.
#include <cuda_runtime.h>

#include <deque>
#include <map>
#include <mutex>
#include <vector>

#include "engine.h"

namespace sdfgpu {

namespace {

// Size classes: 256 B minimum, then four classes per power of two (at most
// 25 % slack).
size_t SizeClass(size_t bytes) {
  size_t b = std::max<size_t>(bytes, 256);
  int top = 63 - __builtin_clzll(b);
  const int shift = std::max(0, top - 2);
  const size_t unit = size_t{1} << shift;
  return (b + unit - 1) / unit * unit;
}

struct Cache {
  std::mutex mu;
  // (device, class) -> free blocks with the stamp of their release, oldest
  // first; device -1 for pinned host blocks
  std::map<std::pair<int, size_t>, std::deque<std::pair<void*, uint64_t>>> free_blocks;
  std::map<int, size_t> cached_bytes;
  uint64_t stamp{0};
};

Cache& TheCache() {
  // never destroyed: blocks stay valid until the process exits
  static Cache* cache = new Cache;
  return *cache;
}

constexpr size_t kMaxCachedDevice = size_t{8} << 30;
constexpr size_t kMaxCachedHost = size_t{256} << 20;

void Release(int dev, void* p) {
  if (dev < 0) {
    cudaFreeHost(p);
  } else {
    cudaFree(p);
  }
}

void* Take(int dev, size_t cls) {
  Cache& c = TheCache();
  const std::lock_guard<std::mutex> lock(c.mu);
  auto it = c.free_blocks.find({dev, cls});
  if (it == c.free_blocks.end() || it->second.empty()) {
    return nullptr;
  }
  void* p = it->second.back().first;
  it->second.pop_back();
  c.cached_bytes[dev] -= cls;
  return p;
}

/// Caches a released block. Over the limit, the blocks of `dev` released
/// longest ago go first: a workload whose sizes drift (a problem growing
/// frame by frame) leaves blocks of classes it no longer asks for, and the
/// working set of the latest sizes must stay cached.
void Keep(int dev, size_t cls, void* p, size_t limit) {
  Cache& c = TheCache();
  std::vector<void*> victims;
  {
    const std::lock_guard<std::mutex> lock(c.mu);
    if (cls > limit) {
      victims.push_back(p);
    } else {
      while (c.cached_bytes[dev] + cls > limit) {
        auto oldest = c.free_blocks.end();
        for (auto it = c.free_blocks.lower_bound({dev, 0}); it != c.free_blocks.end() && it->first.first == dev;
             ++it) {
          if (!it->second.empty() &&
              (oldest == c.free_blocks.end() || it->second.front().second < oldest->second.front().second)) {
            oldest = it;
          }
        }
        if (oldest == c.free_blocks.end()) {
          break;
        }
        victims.push_back(oldest->second.front().first);
        oldest->second.pop_front();
        c.cached_bytes[dev] -= oldest->first.second;
      }
      c.free_blocks[{dev, cls}].emplace_back(p, ++c.stamp);
      c.cached_bytes[dev] += cls;
    }
  }
  for (void* v : victims) {
    Release(dev, v);
  }
}

/// Releases every cached block of `dev` (before retrying a failed allocation).
void Drop(int dev) {
  Cache& c = TheCache();
  std::vector<void*> blocks;
  {
    const std::lock_guard<std::mutex> lock(c.mu);
    for (auto it = c.free_blocks.begin(); it != c.free_blocks.end();) {
      if (it->first.first == dev) {
        for (const auto& b : it->second) {
          blocks.push_back(b.first);
        }
        it = c.free_blocks.erase(it);
      } else {
        ++it;
      }
    }
    c.cached_bytes[dev] = 0;
  }
  for (void* p : blocks) {
    Release(dev, p);
  }
}

int CurrentDevice() {
  int dev = 0;
  CudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
  return dev;
}

}  // namespace

void* CachedDeviceAlloc(size_t bytes, size_t* got) {
  const int dev = CurrentDevice();
  const size_t cls = SizeClass(bytes);
  *got = cls;
  if (void* p = Take(dev, cls)) {
    return p;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, cls);
  if (e != cudaSuccess) {
    cudaGetLastError();
    Drop(dev);
    e = cudaMalloc(&p, cls);
    if (e != cudaSuccess) {
      cudaGetLastError();
      Fail(SDFGPU_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
  }
  return p;
}

void CachedDeviceFree(void* p, size_t cls) { Keep(CurrentDevice(), cls, p, kMaxCachedDevice); }

void* CachedHostAlloc(size_t bytes, size_t* got) {
  const size_t cls = SizeClass(bytes);
  *got = cls;
  if (void* p = Take(-1, cls)) {
    return p;
  }
  void* p = nullptr;
  CudaCheck(cudaMallocHost(&p, cls), "cudaMallocHost");
  return p;
}

void CachedHostFree(void* p, size_t cls) { Keep(-1, cls, p, kMaxCachedHost); }

}  // namespace sdfgpu
