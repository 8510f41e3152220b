// Stable LSD radix sort of (key, value) pairs, 8-bit digits.
//
// Per digit pass: (1) each 4096-key tile counts its digits in shared memory;
// (2) the digit-major count table (256 x tiles) is prefix-summed, giving each
// (digit, tile) its output offset; (3) each tile ranks its keys stably with
// warp match/ballot counters, stages them in shared memory in digit order and
// writes each digit's run contiguously (coalesced) to its offset.
#include <algorithm>

#include "cmh_internal.cuh"

namespace cmh {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kIPT = 16;
constexpr int kTile = kThreads * kIPT;  // 4096
constexpr int kBins = 256;

template <class K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
  return (uint32_t)(k >> shift) & (kBins - 1);
}

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread (256 threads).
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t *warp_sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = warp_inclusive(v);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kWarps ? warp_sums[lane] : 0;
    uint32_t wi = warp_inclusive(w);
    if (lane < kWarps) warp_sums[lane] = wi - w;
  }
  __syncthreads();
  return inc - v + warp_sums[warp];
}

template <class K>
__global__ void __launch_bounds__(kThreads) k_rs_hist(const K *__restrict__ keys, int64_t n_cap,
                                                      const uint32_t *__restrict__ n_dev,
                                                      int shift, uint32_t *__restrict__ hist,
                                                      int64_t ntiles) {
  __shared__ uint32_t h[kBins];
  const int64_t n = n_dev ? (int64_t)*n_dev : n_cap;
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kTile;
#pragma unroll 4
  for (int j = 0; j < kIPT; j++) {
    int64_t i = base + (int64_t)j * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[digit_of(keys[i], shift)], 1u);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// The scatter pass ranks a 4096-key tile with 512 threads x 8 keys: fewer
// registers per thread than the counting pass's layout, so more warps hide
// the memory latency.
constexpr int kSThreads = 512;
constexpr int kSWarps = kSThreads / 32;
constexpr int kSIPT = kTile / kSThreads;  // 8

template <class K>
struct ScatterSmem {
  K keys[kTile];
  uint32_t vals[kTile];
  uint32_t wcnt[kSWarps][kBins];
  uint32_t dstart[kBins];
  uint32_t gofs[kBins];
  uint32_t warp_sums[kSWarps];
};

template <class K>
__global__ void __launch_bounds__(kSThreads) k_rs_scatter(
    const K *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
    K *__restrict__ keys_out, uint32_t *__restrict__ vals_out, int64_t n_cap,
    const uint32_t *__restrict__ n_dev, int shift, const uint32_t *__restrict__ hist_scan,
    int64_t ntiles) {
  const int64_t n = n_dev ? (int64_t)*n_dev : n_cap;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScatterSmem<K> &sm = *reinterpret_cast<ScatterSmem<K> *>(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kTile;

  for (int i = threadIdx.x; i < kSWarps * kBins; i += kSThreads) (&sm.wcnt[0][0])[i] = 0;
  if (threadIdx.x < kBins) sm.gofs[threadIdx.x] = hist_scan[(int64_t)threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();

  const uint32_t lt_mask = (1u << lane) - 1u;
  K k[kSIPT];
  uint32_t v[kSIPT], rank[kSIPT];
#pragma unroll
  for (int j = 0; j < kSIPT; j++) {
    const int64_t i = base + (int64_t)warp * 32 * kSIPT + j * 32 + lane;
    const bool valid = i < n;
    k[j] = valid ? keys_in[i] : K(0);
    v[j] = valid ? vals_in[i] : 0u;
    const uint32_t d = valid ? digit_of(k[j], shift) : (uint32_t)kBins;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t lt = peers & lt_mask;
    uint32_t c = 0;
    if (valid) c = sm.wcnt[warp][d];
    __syncwarp();
    if (valid && lt == 0) sm.wcnt[warp][d] = c + __popc(peers);
    __syncwarp();
    rank[j] = c + __popc(lt);
  }
  __syncthreads();
  {
    // per digit: exclusive prefix over the warps, then over the digits
    const int d = threadIdx.x;
    uint32_t acc = 0;
    if (d < kBins) {
#pragma unroll
      for (int w = 0; w < kSWarps; w++) {
        uint32_t t = sm.wcnt[w][d];
        sm.wcnt[w][d] = acc;
        acc += t;
      }
    }
    uint32_t inc = warp_inclusive(acc);
    if (lane == 31) sm.warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < kSWarps ? sm.warp_sums[lane] : 0;
      uint32_t wi = warp_inclusive(w);
      if (lane < kSWarps) sm.warp_sums[lane] = wi - w;
    }
    __syncthreads();
    if (d < kBins) sm.dstart[d] = inc - acc + sm.warp_sums[warp];
  }
  __syncthreads();
  const int64_t rem = n - base;
#pragma unroll
  for (int j = 0; j < kSIPT; j++) {
    const int64_t i = base + (int64_t)warp * 32 * kSIPT + j * 32 + lane;
    if (i < n) {
      const uint32_t d = digit_of(k[j], shift);
      const uint32_t lp = sm.dstart[d] + sm.wcnt[warp][d] + rank[j];
      sm.keys[lp] = k[j];
      sm.vals[lp] = v[j];
    }
  }
  __syncthreads();
  const int tile_n = rem < kTile ? (int)rem : kTile;
  for (int q = threadIdx.x; q < tile_n; q += kSThreads) {
    const K key = sm.keys[q];
    const uint32_t d = digit_of(key, shift);
    const uint32_t g = sm.gofs[d] + (uint32_t)q - sm.dstart[d];
    keys_out[g] = key;
    vals_out[g] = sm.vals[q];
  }
}

template <class K>
void radix_sort_impl(K *keys, uint32_t *vals, K *keys_alt, uint32_t *vals_alt, int64_t n,
                     const uint32_t *n_dev, int bits, DevBuf &tmp, DevBuf &scan_tmp,
                     cudaStream_t s) {
  if (n <= 1 || bits <= 0) return;
  const int passes = (bits + 7) / 8;
  const int64_t ntiles = (n + kTile - 1) / kTile;
  const int64_t hn = ntiles * kBins;
  if (hn > 0xffffffffll) fail(CMH_ERR_CAPACITY, "radix sort: too many tiles");
  // layout of tmp: hist | hist_scan | scan scratch (own buffer)
  tmp.ensure((size_t)(2 * hn + 64) * sizeof(uint32_t));
  uint32_t *hist = tmp.as<uint32_t>();
  uint32_t *hist_scan = hist + hn;
  const size_t smem = sizeof(ScatterSmem<K>);
  {
    // once per device, never inside a graph capture
    static bool done[64] = {};
    int dev = 0;
    CMH_CUDA(cudaGetDevice(&dev));
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CMH_CUDA(cudaStreamIsCapturing(s, &cs));
    if (dev < 64 && !done[dev] && cs == cudaStreamCaptureStatusNone) {
      CMH_CUDA(cudaFuncSetAttribute(k_rs_scatter<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
      done[dev] = true;
    }
  }
  K *src_k = keys, *dst_k = keys_alt;
  uint32_t *src_v = vals, *dst_v = vals_alt;
  for (int p = 0; p < passes; p++) {
    const int shift = 8 * p;
    k_rs_hist<K><<<(unsigned)ntiles, kThreads, 0, s>>>(src_k, n, n_dev, shift, hist, ntiles);
    CMH_LAUNCHED();
    exclusive_scan_u32(hist, hist_scan, hn, nullptr, scan_tmp, s);
    k_rs_scatter<K><<<(unsigned)ntiles, kSThreads, smem, s>>>(src_k, src_v, dst_k, dst_v, n,
                                                              n_dev, shift, hist_scan, ntiles);
    CMH_LAUNCHED();
    std::swap(src_k, dst_k);
    std::swap(src_v, dst_v);
  }
  if (src_k != keys) {
    CMH_CUDA(cudaMemcpyAsync(keys, src_k, (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, s));
    CMH_CUDA(cudaMemcpyAsync(vals, src_v, (size_t)n * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, s));
  }
}

}  // namespace

void radix_sort_u64_u32(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt,
                        uint32_t *vals_alt, int64_t n, const uint32_t *n_dev, int bits,
                        DevBuf &tmp, DevBuf &scan_tmp, cudaStream_t s) {
  radix_sort_impl<uint64_t>(keys, vals, keys_alt, vals_alt, n, n_dev, bits, tmp, scan_tmp, s);
}

void radix_sort_u32_u32(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt,
                        uint32_t *vals_alt, int64_t n, const uint32_t *n_dev, int bits,
                        DevBuf &tmp, DevBuf &scan_tmp, cudaStream_t s) {
  radix_sort_impl<uint32_t>(keys, vals, keys_alt, vals_alt, n, n_dev, bits, tmp, scan_tmp, s);
}

}  // namespace cmh
