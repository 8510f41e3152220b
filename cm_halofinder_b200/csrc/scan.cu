// Exclusive prefix sum of uint32 values: tile reduce -> scan of tile sums
// (recursive) -> tile scan with the tile's offset.  256 threads x 16 items.
#include <vector>

#include "cmh_internal.cuh"

namespace cmh {
namespace {

constexpr int kThreads = 256;
constexpr int kIPT = 16;
constexpr int kTile = kThreads * kIPT;  // 4096

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += t;
  }
  return v;
}

// Exclusive scan of one value per thread across the block; *tot = block sum.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *tot) {
  __shared__ uint32_t warp_sums[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = warp_inclusive(v);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kThreads / 32 ? warp_sums[lane] : 0;
    uint32_t wi = warp_inclusive(w);
    if (lane < kThreads / 32) warp_sums[lane] = wi - w;
    if (lane == kThreads / 32 - 1) *tot = wi;
  }
  __syncthreads();
  uint32_t r = inc - v + warp_sums[warp];
  __syncthreads();
  return r;
}

__device__ __forceinline__ void load_items(const uint32_t *in, int64_t n, int64_t base,
                                           uint32_t (&x)[kIPT]) {
  const int64_t i0 = base + (int64_t)threadIdx.x * kIPT;
  if (i0 + kIPT <= n && (((uintptr_t)(in + i0)) & 15) == 0) {
    const uint4 *p = reinterpret_cast<const uint4 *>(in + i0);
#pragma unroll
    for (int q = 0; q < kIPT / 4; q++) {
      uint4 v = p[q];
      x[4 * q] = v.x; x[4 * q + 1] = v.y; x[4 * q + 2] = v.z; x[4 * q + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < kIPT; q++) x[q] = (i0 + q < n) ? in[i0 + q] : 0u;
  }
}

// n_dev (device, may be null): the count actually scanned, at most n; the
// entries past it are taken as 0 and not read or written.
__device__ __forceinline__ int64_t live_count(int64_t n, const uint32_t *n_dev) {
  return n_dev ? min(n, (int64_t)*n_dev) : n;
}

__global__ void __launch_bounds__(kThreads) k_tile_reduce(const uint32_t *in, int64_t n,
                                                          const uint32_t *n_dev,
                                                          uint32_t *sums) {
  __shared__ uint32_t tot;
  n = live_count(n, n_dev);
  uint32_t x[kIPT];
  load_items(in, n, (int64_t)blockIdx.x * kTile, x);
  uint32_t s = 0;
#pragma unroll
  for (int q = 0; q < kIPT; q++) s += x[q];
  block_exclusive(s, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kThreads) k_tile_scan(const uint32_t *in, uint32_t *out,
                                                        int64_t n, const uint32_t *n_dev,
                                                        const uint32_t *offsets,
                                                        uint32_t *total) {
  __shared__ uint32_t tot;
  n = live_count(n, n_dev);
  uint32_t x[kIPT];
  const int64_t base = (int64_t)blockIdx.x * kTile;
  load_items(in, n, base, x);
  uint32_t s = 0;
#pragma unroll
  for (int q = 0; q < kIPT; q++) s += x[q];
  uint32_t run = block_exclusive(s, &tot) + (offsets ? offsets[blockIdx.x] : 0u);
  const int64_t i0 = base + (int64_t)threadIdx.x * kIPT;
  if (i0 + kIPT <= n && (((uintptr_t)(out + i0)) & 15) == 0) {
    uint4 *p = reinterpret_cast<uint4 *>(out + i0);
#pragma unroll
    for (int q = 0; q < kIPT / 4; q++) {
      uint4 v;
      v.x = run; run += x[4 * q];
      v.y = run; run += x[4 * q + 1];
      v.z = run; run += x[4 * q + 2];
      v.w = run; run += x[4 * q + 3];
      p[q] = v;
    }
  } else {
#pragma unroll
    for (int q = 0; q < kIPT; q++) {
      if (i0 + q < n) out[i0 + q] = run;
      run += x[q];
    }
  }
  if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    *total = (offsets ? offsets[blockIdx.x] : 0u) + tot;
}

void scan_level(const uint32_t *in, uint32_t *out, int64_t n, const uint32_t *n_dev,
                uint32_t *total, uint32_t *scratch, cudaStream_t s) {
  const int64_t nt = (n + kTile - 1) / kTile;
  if (nt == 1) {
    k_tile_scan<<<1, kThreads, 0, s>>>(in, out, n, n_dev, nullptr, total);
    CMH_LAUNCHED();
    return;
  }
  uint32_t *sums = scratch;
  uint32_t *sums_scan = scratch + nt;
  k_tile_reduce<<<(unsigned)nt, kThreads, 0, s>>>(in, n, n_dev, sums);
  CMH_LAUNCHED();
  scan_level(sums, sums_scan, nt, nullptr, nullptr, scratch + 2 * nt, s);
  k_tile_scan<<<(unsigned)nt, kThreads, 0, s>>>(in, out, n, n_dev, sums_scan, total);
  CMH_LAUNCHED();
}

}  // namespace

void exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total,
                        DevBuf &tmp, cudaStream_t s, const uint32_t *n_dev) {
  if (n <= 0) {
    if (total) CMH_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), s));
    return;
  }
  int64_t need = 0;
  for (int64_t m = n; m > kTile;) {
    m = (m + kTile - 1) / kTile;
    need += 2 * m;
  }
  tmp.ensure((size_t)(need + 16) * sizeof(uint32_t));
  scan_level(in, out, n, n_dev, total, tmp.as<uint32_t>(), s);
}

}  // namespace cmh
