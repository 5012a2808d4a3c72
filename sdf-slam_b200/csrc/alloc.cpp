// Caching allocators for device and pinned host blocks.
//
// cudaMalloc / cudaFree (and cudaMallocHost / cudaFreeHost) take device-wide
// locks, synchronise and cost milliseconds each; a solve handle holds some
// forty buffers, so creating and destroying handles (one per served request,
// one per end-to-end call) spent more time allocating than solving. Freed
// blocks are kept here, per device and per rounded size, and handed to the
// next allocation of the same size class. A block is only returned by an
// owner whose stream has drained, so a reused block has no work in flight.
// Device blocks come from a stream-ordered memory pool of the library's own
// per device (cudaMallocFromPoolAsync / cudaFreeAsync on one allocator
// stream per device):
// returning an evicted block to the pool does not synchronise the device,
// where cudaFree would stall every stream in flight (the served requests of
// other threads included).
#include <cuda_runtime.h>

#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <vector>

#include "engine.h"
#include "host_pool.h"

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

/// Each pool keeps what it has reserved (up to the process's peak use) until
/// an allocation fails, when the retry path trims it: with a lower release
/// threshold every synchronisation handed memory back to the driver and the
/// next allocations mapped it again.
constexpr uint64_t kPoolKeepBytes = ~uint64_t{0};

/// The library's own memory pool of a device and the stream on which blocks
/// are taken from it and returned; an allocation synchronises that stream,
/// so the block is ready for any stream. A private pool leaves the device's
/// default pool (which the host application may use) as it was.
struct DevicePool {
  cudaMemPool_t pool{nullptr};
  cudaStream_t stream{nullptr};
};

struct PoolTable {
  std::mutex mu;
  std::map<int, DevicePool> pools;
};

PoolTable& ThePools() {
  static PoolTable* t = new PoolTable;  // for the process's life
  return *t;
}

/// The pool of `dev`, or null when the library never allocated there.
DevicePool* FindPool(int dev) {
  PoolTable& t = ThePools();
  const std::lock_guard<std::mutex> lock(t.mu);
  auto it = t.pools.find(dev);
  return it == t.pools.end() || it->second.pool == nullptr ? nullptr : &it->second;
}

/// Created on first use, with device `dev` current.
DevicePool& PoolOf(int dev) {
  PoolTable& t = ThePools();
  const std::lock_guard<std::mutex> lock(t.mu);
  DevicePool& d = t.pools[dev];
  if (d.pool == nullptr) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    CudaCheck(cudaMemPoolCreate(&d.pool, &props), "memory pool");
    uint64_t keep = kPoolKeepBytes;
    CudaCheck(cudaMemPoolSetAttribute(d.pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool release threshold");
    CudaCheck(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking), "allocator stream");
  }
  return d;
}

void Release(int dev, void* p) {
  if (dev < 0) {
    cudaFreeHost(p);
  } else if (DevicePool* pool = FindPool(dev)) {
    // on the block's own device and pool stream, whichever device the
    // caller has current
    int cur = dev;
    cudaGetDevice(&cur);
    if (cur != dev) {
      cudaSetDevice(dev);
    }
    cudaFreeAsync(p, pool->stream);
    if (cur != dev) {
      cudaSetDevice(cur);
    }
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

void* CachedDeviceAlloc(size_t bytes, size_t* got, int* device) {
  const int dev = CurrentDevice();
  const size_t cls = SizeClass(bytes);
  *got = cls;
  if (device != nullptr) {
    *device = dev;
  }
  if (void* p = Take(dev, cls)) {
    return p;
  }
  void* p = nullptr;
  DevicePool& pool = PoolOf(dev);
  const cudaStream_t s = pool.stream;
  cudaError_t e = cudaMallocFromPoolAsync(&p, cls, pool.pool, s);
  if (e == cudaSuccess) {
    e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    // give the cached blocks and the pool's reserve back to the driver, retry
    Drop(dev);
    CudaCheck(cudaStreamSynchronize(s), "allocator stream");
    CudaCheck(cudaMemPoolTrimTo(pool.pool, 0), "pool trim");
    e = cudaMallocFromPoolAsync(&p, cls, pool.pool, s);
    if (e == cudaSuccess) {
      e = cudaStreamSynchronize(s);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      Fail(SDFGPU_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
  }
  return p;
}

void ReleaseCachedDeviceMemory() {
  const int dev = CurrentDevice();
  DevicePool* pool = FindPool(dev);
  if (pool == nullptr) {
    return;  // nothing was allocated on this device
  }
  Drop(dev);
  CudaCheck(cudaStreamSynchronize(pool->stream), "allocator stream");
  CudaCheck(cudaMemPoolTrimTo(pool->pool, 0), "pool trim");
}

void CachedDeviceFree(void* p, size_t cls, int device) { Keep(device, cls, p, kMaxCachedDevice); }

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

namespace {

// Copies below this size go straight from pageable memory (a few MB move
// about as fast either way); larger ones are staged in chunks of kStageBytes.
constexpr size_t kStageThreshold = size_t{4} << 20;
constexpr size_t kStageBytes = size_t{16} << 20;

/// Two pinned staging buffers with an event each (the transfer last
/// enqueued from it). A few such slots serve the process; an upload takes a
/// free one or, when all are busy on other threads, copies from pageable
/// memory instead of waiting.
struct Staging {
  std::mutex mu;
  void* buf[2]{nullptr, nullptr};
  cudaEvent_t done[2]{nullptr, nullptr};
  bool ready{false};
};

constexpr int kStagingSlots = 3;

/// The staging slots of `dev`: their events are recorded on that device's
/// streams only (an event and the stream it is recorded on must share a
/// device).
Staging* TheStaging(int dev) {
  static std::mutex mu;
  static std::map<int, Staging*>* slots = new std::map<int, Staging*>;  // kept for the life of the process
  const std::lock_guard<std::mutex> lock(mu);
  Staging*& st = (*slots)[dev];
  if (st == nullptr) {
    st = new Staging[kStagingSlots];
  }
  return st;
}

}  // namespace

void UploadAsync(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes < kStageThreshold) {
    CudaCheck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "upload");
    return;
  }
  Staging* slots = TheStaging(CurrentDevice());
  int slot = -1;
  for (int k = 0; k < kStagingSlots && slot < 0; ++k) {
    if (slots[k].mu.try_lock()) {
      slot = k;
    }
  }
  if (slot < 0) {
    CudaCheck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "upload");
    return;
  }
  Staging& st = slots[slot];
  const std::lock_guard<std::mutex> lock(st.mu, std::adopt_lock);
  if (!st.ready) {
    for (int b = 0; b < 2; ++b) {
      CudaCheck(cudaMallocHost(&st.buf[b], kStageBytes), "staging buffer");
      CudaCheck(cudaEventCreateWithFlags(&st.done[b], cudaEventDisableTiming), "staging event");
    }
    st.ready = true;
  }
  const auto* from = static_cast<const char*>(src);
  auto* to = static_cast<char*>(dst);
  for (size_t off = 0, k = 0; off < bytes; off += kStageBytes, ++k) {
    const size_t len = std::min(kStageBytes, bytes - off);
    const int b = static_cast<int>(k & 1);
    // the buffer's previous transfer has read it
    CudaCheck(cudaEventSynchronize(st.done[b]), "staging wait");
    // filled by the host pool's threads (inline when the pool is busy)
    char* stage = static_cast<char*>(st.buf[b]);
    constexpr size_t kPiece = size_t{2} << 20;
    const int pieces = static_cast<int>((len + kPiece - 1) / kPiece);
    PoolRun(pieces, [&](int p) {
      const size_t a = static_cast<size_t>(p) * kPiece;
      std::memcpy(stage + a, from + off + a, std::min(kPiece, len - a));
    });
    CudaCheck(cudaMemcpyAsync(to + off, st.buf[b], len, cudaMemcpyHostToDevice, s), "upload");
    CudaCheck(cudaEventRecord(st.done[b], s), "staging event");
  }
}

}  // namespace sdfgpu
