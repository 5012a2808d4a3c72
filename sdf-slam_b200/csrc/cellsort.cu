// Stable LSD radix sort of point rows by grid cell.
//
// The J^T J column gather needs, for every cell, the point rows that fall in
// it in ascending row order (the reference accumulates each J^T J entry in
// ascending row order, src/solvers/lm_solver.cpp:113-172). Rows arrive in
// row order, so a stable sort on the cell key alone gives that order.
// 8-bit digits; per pass: a per-tile digit histogram, one exclusive scan over
// (digit, tile) (KDigitScan), and a stable scatter that ranks equal digits inside a warp
// with __match_any_sync and across warps with shared counters.
#include <cuda_runtime.h>

#include "device.cuh"

namespace sdfgpu {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per block

__global__ void KRadixHist(const int32_t* keys, int64_t n, int shift, int32_t* hist, int num_tiles) {
  __shared__ int32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kSortTile;
  for (int q = 0; q < kSortItems; ++q) {
    const int64_t idx = base + q * kSortThreads + threadIdx.x;
    if (idx < n) {
      atomicAdd(&h[(static_cast<uint32_t>(keys[idx]) >> shift) & 255u], 1);
    }
  }
  __syncthreads();
  hist[static_cast<int64_t>(threadIdx.x) * num_tiles + blockIdx.x] = h[threadIdx.x];
}

/// Exclusive scan, in place, of the digit histogram hist[digit * tiles +
/// tile] in (digit, tile) order, by one block of 1024 threads: warp w owns
/// digits 8w..8w+7 and walks their rows in chunks of 32 tiles (lane = tile,
/// coalesced, the eight rows' loads in flight together). Pass one sums each
/// row, a scan of the 256 row totals gives every digit's start, pass two
/// scans each row chunk by chunk with a carry.
__global__ void __launch_bounds__(1024) KDigitScan(int32_t* hist, int tiles) {
  __shared__ int32_t start[256];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int32_t* rows = hist + static_cast<int64_t>(8 * warp) * tiles;
  int32_t sum[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    sum[i] = 0;
  }
#pragma unroll 2
  for (int c0 = 0; c0 < tiles; c0 += 32) {
    const int t = c0 + lane;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      sum[i] += t < tiles ? rows[static_cast<int64_t>(i) * tiles + t] : 0;
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      sum[i] += __shfl_xor_sync(0xffffffffu, sum[i], d);
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      start[8 * warp + i] = sum[i];
    }
  }
  __syncthreads();
  if (warp == 0) {
    // exclusive scan of the 256 totals: lane l owns digits 8l..8l+7
    int32_t v[8];
    int32_t own = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      v[i] = start[8 * lane + i];
      own += v[i];
    }
    int32_t x = own;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) {
        x += y;
      }
    }
    int32_t run = x - own;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      start[8 * lane + i] = run;
      run += v[i];
    }
  }
  __syncthreads();
  int32_t carry[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    carry[i] = start[8 * warp + i];
  }
  for (int c0 = 0; c0 < tiles; c0 += 32) {
    const int t = c0 + lane;
    int32_t v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      v[i] = t < tiles ? rows[static_cast<int64_t>(i) * tiles + t] : 0;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int32_t x = v[i];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) {
          x += y;
        }
      }
      if (t < tiles) {
        rows[static_cast<int64_t>(i) * tiles + t] = carry[i] + x - v[i];
      }
      carry[i] += __shfl_sync(0xffffffffu, x, 31);
    }
  }
}

__global__ void KRadixScatter(const int32_t* keys_in, const int32_t* vals_in, int64_t n, int shift,
                              const int32_t* offsets, int num_tiles, int32_t* keys_out, int32_t* vals_out) {
  __shared__ int32_t wcount[kSortThreads / 32][256];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int d = lane; d < 256; d += 32) {
    wcount[warp][d] = 0;
  }
  __syncwarp();
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kSortTile + static_cast<int64_t>(warp) * (32 * kSortItems);
  int rank[kSortItems];
  int digit[kSortItems];
  int32_t key[kSortItems];
  int32_t val[kSortItems];
  const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const int64_t idx = base + q * 32 + lane;
    const bool ok = idx < n;
    key[q] = ok ? keys_in[idx] : 0;
    val[q] = ok ? vals_in[idx] : 0;
    const int d = ok ? static_cast<int>((static_cast<uint32_t>(key[q]) >> shift) & 255u) : 256 + lane;
    digit[q] = d;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    int before = 0;
    if (ok) {
      before = wcount[warp][d];
    }
    __syncwarp();
    rank[q] = before + __popc(peers & lt_mask);
    if (ok && lane == leader) {
      wcount[warp][d] = before + __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  {
    const int d = threadIdx.x;  // 256 threads, one per digit
    int running = 0;
    for (int w = 0; w < kSortThreads / 32; ++w) {
      const int c = wcount[w][d];
      wcount[w][d] = running;
      running += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kSortItems; ++q) {
    const int64_t idx = base + q * 32 + lane;
    if (idx < n) {
      const int d = digit[q];
      const int64_t pos = static_cast<int64_t>(offsets[static_cast<int64_t>(d) * num_tiles + blockIdx.x]) +
                          wcount[warp][d] + rank[q];
      keys_out[pos] = key[q];
      vals_out[pos] = val[q];
    }
  }
}

/// Keys: cell of each point row (invalid rows get the sentinel num_cells);
/// values: row ids.
__global__ void KCellKeys(const int32_t* pt_cell, int64_t n, int32_t sentinel, int32_t* keys, int32_t* vals) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k < n) {
    const int32_t c = pt_cell[k];
    keys[k] = c < 0 ? sentinel : c;
    vals[k] = static_cast<int32_t>(k);
  }
}

/// Host launcher: sorts (pt_cell, row) pairs; result rows in vals_a / keys_a
/// (ping-pong buffers of n entries each; hist of 256 * tiles entries).
void LaunchCellSort(const int32_t* pt_cell, int64_t n, int64_t num_cells, int32_t* keys_a, int32_t* vals_a,
                    int32_t* keys_b, int32_t* vals_b, int32_t* hist, cudaStream_t stream, bool* result_in_a) {
  const int tiles = static_cast<int>((n + kSortTile - 1) / kSortTile);
  KCellKeys<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(pt_cell, n, static_cast<int32_t>(num_cells),
                                                                         keys_a, vals_a);
  int bits = 1;
  while ((int64_t{1} << bits) <= num_cells) {
    ++bits;
  }
  int32_t* kin = keys_a;
  int32_t* vin = vals_a;
  int32_t* kout = keys_b;
  int32_t* vout = vals_b;
  bool in_a = true;
  for (int shift = 0; shift < bits; shift += 8) {
    KRadixHist<<<tiles, kSortThreads, 0, stream>>>(kin, n, shift, hist, tiles);
    KDigitScan<<<1, 1024, 0, stream>>>(hist, tiles);
    KRadixScatter<<<tiles, kSortThreads, 0, stream>>>(kin, vin, n, shift, hist, tiles, kout, vout);
    std::swap(kin, kout);
    std::swap(vin, vout);
    in_a = !in_a;
  }
  *result_in_a = in_a;
}

}  // namespace sdfgpu
