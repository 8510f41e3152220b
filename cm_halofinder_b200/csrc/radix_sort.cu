// Stable LSD radix sort of (key, value) pairs, 8-bit digits.
//
// One read of the keys counts the digits of every pass (k_rs_upfront), which
// gives each digit's start in the output.  Each pass is then a single
// kernel: each 4096-key tile ranks its keys stably with warp match/ballot
// counters, learns how many keys of each digit the lower tiles hold by
// decoupled look-back over published tile states, stages its keys in shared
// memory in digit order and writes each digit's run contiguously
// (coalesced).  A sort of 64-bit keys whose sorted keys are not wanted
// narrows them to 32-bit words at the first pass after which at most 32 key
// bits remain (the consumed low digits are dropped), so that the later
// passes move 8 bytes per pair instead of 12; and those 32-bit passes use
// 9-bit digits where that saves a pass (26 bits: 9 + 9 + 8, not 8 + 8 + 8 + 2).
#include <algorithm>

#include "cmh_internal.cuh"

namespace cmh {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kIPT = 16;
constexpr int kTile = kThreads * kIPT;  // 4096
constexpr int kBins = 256;      // 8-bit digits
constexpr int kMaxBins = 512;   // 9-bit digits
constexpr int kMaxPasses = 8;
// Tile states of the look-back, one 64-bit word per (tile, digit): the flag
// in the high half, the count in the low half, written in one store.
constexpr uint64_t kAggregate = 1ull << 32;  // count = the tile's own keys of the digit
constexpr uint64_t kInclusive = 2ull << 32;  // count = keys of the digit up to this tile

template <int BINS = kBins, class K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
  return (uint32_t)(k >> shift) & (BINS - 1);
}

// The digits of a sort's passes: shift in the original key and width (8 or
// 9 bits).
struct PassDigits {
  int passes;
  int shift[kMaxPasses];
  int width[kMaxPasses];
};

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += t;
  }
  return v;
}


// All digit histograms of the sort in one read of the keys: pass p's
// counters at ghist[kMaxBins p].
template <class K>
__global__ void __launch_bounds__(kThreads) k_rs_upfront(const K *__restrict__ keys,
                                                         int64_t n_cap,
                                                         const uint32_t *__restrict__ n_dev,
                                                         PassDigits pd,
                                                         uint32_t *__restrict__ ghist) {
  __shared__ uint32_t h[kMaxPasses * kMaxBins];
  const int64_t n = n_dev ? (int64_t)*n_dev : n_cap;
  for (int i = threadIdx.x; i < pd.passes * kMaxBins; i += kThreads) h[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * kThreads) {
    const K k = keys[i];
    for (int p = 0; p < pd.passes; p++)
      atomicAdd(&h[p * kMaxBins + ((uint32_t)(k >> pd.shift[p]) & ((1u << pd.width[p]) - 1u))],
                1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < pd.passes * kMaxBins; i += kThreads)
    if (h[i]) atomicAdd(&ghist[i], h[i]);
}

// Exclusive prefix over the digits of each pass (one CTA of kMaxBins
// threads per pass; unused digits count 0).
__global__ void __launch_bounds__(kMaxBins) k_rs_offsets(const uint32_t *__restrict__ ghist,
                                                         uint32_t *__restrict__ goff) {
  __shared__ uint32_t warp_sums[kMaxBins / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t v = ghist[blockIdx.x * kMaxBins + threadIdx.x];
  const uint32_t inc = warp_inclusive(v);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = lane < kMaxBins / 32 ? warp_sums[lane] : 0;
    const uint32_t wi = warp_inclusive(w);
    if (lane < kMaxBins / 32) warp_sums[lane] = wi - w;
  }
  __syncthreads();
  goff[blockIdx.x * kMaxBins + threadIdx.x] = inc - v + warp_sums[warp];
}

// One digit pass, single sweep: a CTA takes the next tile from a counter
// (so every lower tile is already being worked on), ranks its 4096 keys
// stably in shared memory (512 threads x 8 keys; warp match/ballot counters),
// publishes its per-digit counts, then finds the counts of all lower tiles
// by looking back through their published states (decoupled look-back:
// inclusive states end the walk) and writes each digit's run contiguously to
// goff[digit] + (keys of the digit in lower tiles).  A tile publishes its own
// counts before it waits on anything, so every wait ends; a wait is still
// capped, and a capped one sets *giveups.
constexpr int kSThreads = 512;
constexpr int kSWarps = kSThreads / 32;
constexpr int kSIPT = kTile / kSThreads;  // 8

template <class K, int BINS>
struct ScatterSmem {
  K keys[kTile];
  uint32_t vals[kTile];
  uint32_t wcnt[kSWarps][BINS];
  uint32_t dstart[BINS];
  uint32_t gofs[BINS];
  uint32_t thist[BINS];
  uint32_t warp_sums[kSWarps];
  uint32_t tile;
};

// Lanes of the warp with the same NB-bit value d (a digit, or BINS for an
// empty slot): one ballot per bit.
template <int NB>
__device__ __forceinline__ uint32_t peers_of(uint32_t d) {
  uint32_t peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const uint32_t m = __ballot_sync(0xffffffffu, (d >> b) & 1u);
    peers &= ((d >> b) & 1u) ? m : ~m;
  }
  return peers;
}

__device__ __forceinline__ uint64_t load_state(const uint64_t *p) {
  return *reinterpret_cast<const volatile uint64_t *>(p);
}

// Keys are read as K and written as KO = K >> out_shift (out_shift 0 unless
// the pass narrows 64-bit keys to 32 bits); digits have log2(BINS) bits.
// With 32-bit keys and 8-bit digits a CTA's shared memory is small enough for
// 4 CTAs per SM.
template <class K, class KO, int BINS>
__global__ void __launch_bounds__(kSThreads, (sizeof(K) == 4 && BINS == BINS) ? 4 : 3) k_rs_scatter(
    const K *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
    KO *__restrict__ keys_out, uint32_t *__restrict__ vals_out, int64_t n_cap,
    const uint32_t *__restrict__ n_dev, int shift, int out_shift,
    const uint32_t *__restrict__ goff,
    uint64_t *__restrict__ state, uint32_t *__restrict__ tile_ctr,
    unsigned int *__restrict__ giveups, SortWaits waits) {
  const int64_t n = n_dev ? (int64_t)*n_dev : n_cap;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ScatterSmem<K, BINS> &sm = *reinterpret_cast<ScatterSmem<K, BINS> *>(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) sm.tile = atomicAdd(tile_ctr, 1u);
  for (int i = threadIdx.x; i < kSWarps * BINS; i += kSThreads) (&sm.wcnt[0][0])[i] = 0;
  if (threadIdx.x < BINS) sm.thist[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t tile = sm.tile;
  const int64_t base = (int64_t)tile * kTile;
  if (base >= n) return;  // the whole CTA leaves together
  const uint32_t lt_mask = (1u << lane) - 1u;
  K k[kSIPT];
  uint32_t v[kSIPT], rank[kSIPT];
#pragma unroll
  for (int j = 0; j < kSIPT; j++) {
    const int64_t i = base + (int64_t)warp * 32 * kSIPT + j * 32 + lane;
    const bool valid = i < n;
    k[j] = valid ? keys_in[i] : K(0);
    v[j] = valid ? vals_in[i] : 0u;
  }
  // the tile's digit counts first, published before the ranking so that
  // the higher tiles' look-back finds them early
#pragma unroll
  for (int j = 0; j < kSIPT; j++)
    if (base + (int64_t)warp * 32 * kSIPT + j * 32 + lane < n)
      atomicAdd(&sm.thist[digit_of<BINS>(k[j], shift)], 1u);
  __syncthreads();
  // (a tile named by waits.stall_tile publishes nothing: a test hook whose
  // successor's capped wait then runs out)
  if (threadIdx.x < BINS && tile != waits.stall_tile)
    atomicExch(reinterpret_cast<unsigned long long *>(state + (uint64_t)tile * BINS + threadIdx.x),
               (unsigned long long)((tile == 0 ? kInclusive : kAggregate) | sm.thist[threadIdx.x]));
#pragma unroll
  for (int j = 0; j < kSIPT; j++) {
    const int64_t i = base + (int64_t)warp * 32 * kSIPT + j * 32 + lane;
    const bool valid = i < n;
    const uint32_t d = valid ? digit_of<BINS>(k[j], shift) : (uint32_t)BINS;
    const uint32_t peers = peers_of<BINS == 512 ? 10 : 9>(d);
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
    if (d < BINS) {
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
    if (d < BINS) {
      sm.dstart[d] = inc - acc + sm.warp_sums[warp];
      // add up the lower tiles' counts, then publish the running total
      uint64_t *mine = state + (uint64_t)tile * BINS + d;
      uint32_t excl = 0;
      if (tile != 0) {
        for (int64_t j = (int64_t)tile - 1; j >= 0; j--) {
          const uint64_t *p = state + (uint64_t)j * BINS + d;
          uint64_t w = load_state(p);
          for (uint32_t spin = 0; (w >> 32) == 0 && spin < waits.spin_cap; spin++)
            w = load_state(p);
          if ((w >> 32) == 0) {
            atomicAdd(giveups, 1u);
            break;
          }
          excl += (uint32_t)w;
          if ((w >> 32) == 2) break;
        }
        if (tile != waits.stall_tile)
          atomicExch(reinterpret_cast<unsigned long long *>(mine),
                     (unsigned long long)(kInclusive | (uint64_t)(excl + acc)));
      }
      sm.gofs[d] = goff[d] + excl;
    }
  }
  __syncthreads();
  const int64_t rem = n - base;
#pragma unroll
  for (int j = 0; j < kSIPT; j++) {
    const int64_t i = base + (int64_t)warp * 32 * kSIPT + j * 32 + lane;
    if (i < n) {
      const uint32_t d = digit_of<BINS>(k[j], shift);
      const uint32_t lp = sm.dstart[d] + sm.wcnt[warp][d] + rank[j];
      sm.keys[lp] = k[j];
      sm.vals[lp] = v[j];
    }
  }
  __syncthreads();
  const int tile_n = rem < kTile ? (int)rem : kTile;
  for (int q = threadIdx.x; q < tile_n; q += kSThreads) {
    const K key = sm.keys[q];
    const uint32_t d = digit_of<BINS>(key, shift);
    const uint32_t g = sm.gofs[d] + (uint32_t)q - sm.dstart[d];
    keys_out[g] = (KO)(key >> out_shift);
    vals_out[g] = sm.vals[q];
  }
}

// Dynamic shared memory of every scatter instantiation, set once per device
// (never inside a graph capture).
void set_scatter_smem(cudaStream_t s) {
  static bool done[64] = {};
  int dev = 0;
  CMH_CUDA(cudaGetDevice(&dev));
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CMH_CUDA(cudaStreamIsCapturing(s, &cs));
  if (dev >= 64 || done[dev] || cs != cudaStreamCaptureStatusNone) return;
  CMH_CUDA(cudaFuncSetAttribute(k_rs_scatter<uint64_t, uint64_t, kBins>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ScatterSmem<uint64_t, kBins>)));
  CMH_CUDA(cudaFuncSetAttribute(k_rs_scatter<uint64_t, uint32_t, kBins>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ScatterSmem<uint64_t, kBins>)));
  CMH_CUDA(cudaFuncSetAttribute(k_rs_scatter<uint32_t, uint32_t, kBins>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ScatterSmem<uint32_t, kBins>)));
  CMH_CUDA(cudaFuncSetAttribute(k_rs_scatter<uint32_t, uint32_t, kMaxBins>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ScatterSmem<uint32_t, kMaxBins>)));
  done[dev] = true;
}

// The passes of a sort of `bits`-bit keys.  Plain: 8-bit digits.  Narrowed:
// m 8-bit passes over the 64-bit keys, m the fewest after which at most 32
// bits remain, then the 32-bit passes over the R bits left, with 9-bit
// digits on the first R - 8 ceil(R / 9) of them when that takes fewer passes
// than 8-bit digits.  *wide receives m.
PassDigits plan_passes(int bits, bool narrow, int *wide) {
  PassDigits pd{};
  int m = (bits + 7) / 8, nine = 0, q = 0;
  if (narrow) {
    m = std::min((bits + 7) / 8, std::max(1, (bits - 32 + 7) / 8));
    const int rest = std::max(0, bits - 8 * m);
    const int q8 = (rest + 7) / 8, q9 = (rest + 8) / 9;
    q = q9 < q8 ? q9 : q8;
    nine = q9 < q8 ? rest - 8 * q9 : 0;
  }
  pd.passes = m + q;
  int shift = 0;
  for (int p = 0; p < pd.passes; p++) {
    pd.shift[p] = shift;
    pd.width[p] = (p >= m && p - m < nine) ? 9 : 8;
    shift += pd.width[p];
  }
  *wide = m;
  return pd;
}

// With `narrow` (64-bit keys whose sorted order, not their sorted copy, is
// wanted) the first m passes read 64-bit keys; pass m-1 writes key >> 8m as
// 32-bit words and the later passes sort those on the digits that are left.
template <class K>
void radix_sort_impl(K *keys, uint32_t *vals, K *keys_alt, uint32_t *vals_alt, int64_t n,
                     const uint32_t *n_dev, int bits, DevBuf &tmp, unsigned int *giveups,
                     cudaStream_t s, bool copy_back, bool narrow, SortWaits waits) {
  if (bits <= 0) return;
  if (bits > (int)(8 * sizeof(K)) || (bits + 7) / 8 > kMaxPasses)
    fail(CMH_ERR_INVALID_ARGUMENT, "radix sort: key bits out of range");
  if (narrow && (copy_back || sizeof(K) != 8))
    fail(CMH_ERR_INVALID_ARGUMENT, "radix sort: narrowing applies to 64-bit keys left unsorted");
  int m = 0;
  const PassDigits pd = plan_passes(bits, narrow, &m);
  const int passes = pd.passes;
  if (n <= 1) {
    // nothing to order; still leave the data where the caller expects it
    if (!copy_back && passes % 2 == 1 && n == 1) {
      CMH_CUDA(cudaMemcpyAsync(keys_alt, keys, sizeof(K), cudaMemcpyDeviceToDevice, s));
      CMH_CUDA(cudaMemcpyAsync(vals_alt, vals, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    }
    return;
  }
  const int64_t ntiles = (n + kTile - 1) / kTile;
  if (ntiles >= 0xffffffffll) fail(CMH_ERR_CAPACITY, "radix sort: too many tiles");
  // tmp: tile states (ntiles x 512 u64) | digit counts | digit offsets | tile counters
  const size_t state_bytes = (size_t)ntiles * kMaxBins * sizeof(uint64_t);
  const size_t small = (size_t)(2 * kMaxPasses * kMaxBins + kMaxPasses) * sizeof(uint32_t);
  tmp.ensure(radix_sort_scratch(n));
  uint64_t *state = tmp.as<uint64_t>();
  uint32_t *ghist = reinterpret_cast<uint32_t *>(tmp.as<unsigned char>() + state_bytes);
  uint32_t *goff = ghist + kMaxPasses * kMaxBins;
  uint32_t *tile_ctr = goff + kMaxPasses * kMaxBins;
  set_scatter_smem(s);
  CMH_CUDA(cudaMemsetAsync(ghist, 0, small, s));
  k_rs_upfront<K><<<grid_resident(reinterpret_cast<const void *>(k_rs_upfront<K>), kThreads, 0,
                                  n),
                    kThreads, 0, s>>>(keys, n, n_dev, pd, ghist);
  CMH_LAUNCHED();
  k_rs_offsets<<<passes, kMaxBins, 0, s>>>(ghist, goff);
  CMH_LAUNCHED();
  void *src_k = keys, *dst_k = keys_alt;
  uint32_t *src_v = vals, *dst_v = vals_alt;
  for (int p = 0; p < passes; p++) {
    const int bins = 1 << pd.width[p];
    CMH_CUDA(cudaMemsetAsync(state, 0, (size_t)ntiles * bins * sizeof(uint64_t), s));
    const uint32_t *go = goff + p * kMaxBins;
    // the stall hook applies to the first pass only
    const SortWaits wp{waits.spin_cap, p == 0 ? waits.stall_tile : 0xffffffffu};
    if (p < m && !(narrow && p == m - 1)) {
      k_rs_scatter<K, K, kBins><<<(unsigned)ntiles, kSThreads, sizeof(ScatterSmem<K, kBins>), s>>>(
          static_cast<const K *>(src_k), src_v, static_cast<K *>(dst_k), dst_v, n, n_dev,
          pd.shift[p], 0, go, state, tile_ctr + p, giveups, wp);
    } else if (p < m) {
      k_rs_scatter<K, uint32_t, kBins>
          <<<(unsigned)ntiles, kSThreads, sizeof(ScatterSmem<K, kBins>), s>>>(
              static_cast<const K *>(src_k), src_v, static_cast<uint32_t *>(dst_k), dst_v, n,
              n_dev, pd.shift[p], 8 * m, go, state, tile_ctr + p, giveups, wp);
    } else if (bins == kMaxBins) {
      k_rs_scatter<uint32_t, uint32_t, kMaxBins>
          <<<(unsigned)ntiles, kSThreads, sizeof(ScatterSmem<uint32_t, kMaxBins>), s>>>(
              static_cast<const uint32_t *>(src_k), src_v, static_cast<uint32_t *>(dst_k), dst_v,
              n, n_dev, pd.shift[p] - 8 * m, 0, go, state, tile_ctr + p, giveups, wp);
    } else {
      k_rs_scatter<uint32_t, uint32_t, kBins>
          <<<(unsigned)ntiles, kSThreads, sizeof(ScatterSmem<uint32_t, kBins>), s>>>(
              static_cast<const uint32_t *>(src_k), src_v, static_cast<uint32_t *>(dst_k), dst_v,
              n, n_dev, pd.shift[p] - 8 * m, 0, go, state, tile_ctr + p, giveups, wp);
    }
    CMH_LAUNCHED();
    std::swap(src_k, dst_k);
    std::swap(src_v, dst_v);
  }
  if (src_k != keys && copy_back) {
    CMH_CUDA(cudaMemcpyAsync(keys, src_k, (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, s));
    CMH_CUDA(cudaMemcpyAsync(vals, src_v, (size_t)n * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, s));
  }
}

}  // namespace

size_t radix_sort_scratch(int64_t n) {
  const int64_t ntiles = (std::max<int64_t>(n, 1) + kTile - 1) / kTile;
  return (size_t)ntiles * kMaxBins * sizeof(uint64_t) +
         (size_t)(2 * kMaxPasses * kMaxBins + kMaxPasses) * sizeof(uint32_t);
}

int radix_order_passes(int bits) {
  int m = 0;
  return bits > 0 ? plan_passes(bits, true, &m).passes : 0;
}

void radix_sort_u64_u32(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt,
                        uint32_t *vals_alt, int64_t n, const uint32_t *n_dev, int bits,
                        DevBuf &tmp, unsigned int *giveups, cudaStream_t s, bool copy_back,
                        SortWaits waits) {
  radix_sort_impl<uint64_t>(keys, vals, keys_alt, vals_alt, n, n_dev, bits, tmp, giveups, s,
                            copy_back, false, waits);
}

void radix_order_u64_u32(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt,
                         uint32_t *vals_alt, int64_t n, const uint32_t *n_dev, int bits,
                         DevBuf &tmp, unsigned int *giveups, cudaStream_t s, SortWaits waits) {
  radix_sort_impl<uint64_t>(keys, vals, keys_alt, vals_alt, n, n_dev, bits, tmp, giveups, s,
                            false, true, waits);
}

void radix_sort_u32_u32(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt,
                        uint32_t *vals_alt, int64_t n, const uint32_t *n_dev, int bits,
                        DevBuf &tmp, unsigned int *giveups, cudaStream_t s, SortWaits waits) {
  radix_sort_impl<uint32_t>(keys, vals, keys_alt, vals_alt, n, n_dev, bits, tmp, giveups, s,
                            true, false, waits);
}

}  // namespace cmh
