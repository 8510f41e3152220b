// Internal declarations of the B200 FoF library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/cmh_fof.h"

namespace cmh {

constexpr int kSMs = 148;  // B200: 2 dies x 74 SMs

// Per-thread error message behind cmh_last_error().
void set_error(const std::string &msg);

struct Error {
  cmh_status code;
  std::string msg;
};

// Throws Error on a CUDA failure; the C ABI layer turns it into a status.
void cuda_check(cudaError_t e, const char *what, const char *file, int line);
#define CMH_CUDA(x) ::cmh::cuda_check((x), #x, __FILE__, __LINE__)

// Kernels launched by this host thread (reported per run in cmh_stats).
extern thread_local long long g_launches;
#define CMH_LAUNCHED()                     \
  do {                                     \
    CMH_CUDA(cudaGetLastError());          \
    ++::cmh::g_launches;                   \
  } while (0)
[[noreturn]] void fail(cmh_status code, const std::string &msg);

// Host-side fault injection for tests: whether `kind` is one of the
// comma-separated words of the CMH_FAULT environment variable (alloc: device
// allocations fail; io: opening a file fails; overflow: every run overflows
// its capacity; lookback: one tile of the cell sort publishes nothing, so a
// capped device wait runs out).  Read on every call, in host code only.
bool fault_active(const char *kind);

// Grid size for a grid-stride kernel: a multiple of the SM count, capped by
// the work.
inline unsigned grid_for(int64_t n, int threads, int per_sm = 8) {
  int64_t want = (n + threads - 1) / threads;
  int64_t cap = (int64_t)kSMs * per_sm;
  if (want < 1) want = 1;
  return (unsigned)(want < cap ? want : cap);
}

// CTAs of `kernel` (with `threads` threads and `smem` bytes of dynamic shared
// memory) resident at once on the current device: per-SM occupancy times the
// SM count, cached per kernel, shape and device.
int resident_ctas(const void *kernel, int threads, size_t smem);

// Grid for a grid-stride kernel: one resident wave, capped by the work.
inline unsigned grid_resident(const void *kernel, int threads, size_t smem, int64_t n) {
  int64_t want = (n + threads - 1) / threads;
  const int64_t cap = resident_ctas(kernel, threads, smem);
  if (want < 1) want = 1;
  return (unsigned)(want < cap ? want : cap);
}

// Growable device buffer.
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  void ensure(size_t bytes);
  void release();
  template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

// ---- scan.cu ---------------------------------------------------------------
// Exclusive prefix sum of n uint32 values; `total` (device, may be null)
// receives the sum.  Scratch is taken from `tmp` (grown as needed).  With
// `n_dev` (device) only the first min(n, *n_dev) entries are read and
// written; n sizes the launches.
void exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n,
                        uint32_t *total, DevBuf &tmp, cudaStream_t s,
                        const uint32_t *n_dev = nullptr);

// ---- radix_sort.cu -----------------------------------------------------------
// Bounds of the sorts' look-back waits: a tile polls a lower tile's state at
// most spin_cap times, then gives up (the sort's giveups counter is raised;
// its output is then not an ordering).  stall_tile (a test hook) names a tile
// of the first pass that publishes nothing, so that its successor's wait
// runs out.
constexpr uint32_t kSpinCap = 1u << 22;
struct SortWaits {
  uint32_t spin_cap = kSpinCap;
  uint32_t stall_tile = 0xffffffffu;
};

// Stable LSD radix sort of (key u64, value u32) pairs on the low `bits` key
// bits.  Result lands in keys/vals (the alt buffers are scratch); `tmp`
// holds the digit counts and the tiles' look-back states.
// `n` sizes the launches; with `n_dev` set, the element count is read from
// device memory (at most n), so the sort needs no host synchronisation.
// `tmp` must already hold radix_sort_scratch(n) bytes when the sort is
// captured in a graph; `giveups` (device) counts capped look-back waits.
// With copy_back false and an odd number of 8-bit passes the result stays in
// keys_alt/vals_alt (no copy).
void radix_sort_u64_u32(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt,
                        uint32_t *vals_alt, int64_t n, const uint32_t *n_dev, int bits,
                        DevBuf &tmp, unsigned int *giveups, cudaStream_t s,
                        bool copy_back = true, SortWaits waits = SortWaits{});
// The values of the same sort, in key order, without the sorted keys: both
// key buffers end as scratch (the later passes move 32-bit key words, with
// 9-bit digits where that saves a pass), and the values end in vals_alt
// after an odd number of passes (radix_order_passes), else in vals.
int radix_order_passes(int bits);
void radix_order_u64_u32(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt,
                         uint32_t *vals_alt, int64_t n, const uint32_t *n_dev, int bits,
                         DevBuf &tmp, unsigned int *giveups, cudaStream_t s,
                         SortWaits waits = SortWaits{});
// Same for 32-bit keys.
void radix_sort_u32_u32(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt,
                        uint32_t *vals_alt, int64_t n, const uint32_t *n_dev, int bits,
                        DevBuf &tmp, unsigned int *giveups, cudaStream_t s,
                        SortWaits waits = SortWaits{});
// Scratch bytes of a sort of up to n keys.
size_t radix_sort_scratch(int64_t n);

}  // namespace cmh
