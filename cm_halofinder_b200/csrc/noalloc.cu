// FoF group labels for small particle sets without any device allocation.
//
// Some callers cannot call cudaMalloc: a process whose framework has already
// reserved nearly all device memory for its own caching allocator, a service
// that forbids allocation after start-up so that latency stays flat, or a
// plugin host that only lends out buffers it owns.  For them this variant
// keeps its scratch -- union-find parents, cell lists and error flags -- in
// one file-scope device array of fixed size that every GPU loading the
// library holds until the process exits.  The caller still passes the input
// positions and the output label array (device memory it owns).
//
// Limits: at most kMaxParticles particles and a cell grid of at most
// kMaxCells cells (the cell side grows to fit).  Non-periodic only.
//
// Sharing: every call on a device uses the same array.  Each call clears what
// must start empty before use, but two calls whose work overlaps on the GPU
// (for instance on two streams) race on the array and give wrong labels.
#include <cuda.h>

#include <cmath>
#include <mutex>

#include "cmh_internal.cuh"
#include "fof_kernels.cuh"

namespace cmh {
namespace {

constexpr int kMaxParticles = 1 << 16;
constexpr int kMaxCells = 1 << 18;
constexpr int kThreads = 256;

struct NoAllocScratch {
  uint32_t parent[kMaxParticles];
  uint32_t next[kMaxParticles];
  uint32_t cell_head[kMaxCells];
  Counters ctr;         // uf_giveups is the error flag of the union loop
  unsigned int flags[4];  // [0] particles outside the padded domain
};

static __device__ __align__(256) NoAllocScratch g_noalloc;

// Host-side address of g_noalloc on each device, looked up with that device
// current.  In host code the symbol itself is only a stand-in, never a device
// address.  The lookup is redone only when the device's context changed (a
// cudaDeviceReset followed by new work loads the module again, and the array
// may then sit elsewhere); the context is told apart by its ID, which the
// driver never reuses within a process.
std::mutex g_addr_mutex;
struct ScratchAddr {
  NoAllocScratch *p = nullptr;
  unsigned long long ctx_id = 0;
};
ScratchAddr g_addr[128];

// ID of the calling thread's current context, 0 when none is current.
unsigned long long current_context_id() {
  typedef CUresult(CUDAAPI * CtxGetCurrent)(CUcontext *);
  typedef CUresult(CUDAAPI * CtxGetId)(CUcontext, unsigned long long *);
  static CtxGetCurrent get_current = nullptr;
  static CtxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void **)&get_current, cudaEnableDefault,
                                &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
      get_current = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", (void **)&get_id, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess)
      get_id = nullptr;
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

NoAllocScratch *scratch_on(int device) {
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (device < 0 || device >= 128) fail(CMH_ERR_INVALID_ARGUMENT, "device index out of range");
  ScratchAddr &a = g_addr[device];
  const unsigned long long id = current_context_id();
  if (!a.p || id == 0 || id != a.ctx_id) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc);
    if (e != cudaSuccess || !p)
      fail(CMH_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                             cudaGetErrorString(e));
    a.p = static_cast<NoAllocScratch *>(p);
    a.ctx_id = current_context_id();  // the lookup made the primary context current
  }
  return a.p;
}

struct NaGrid {
  double rmin[3], lc;
  int nc[3];
  double rmax[3];
  double linksq;
};

__global__ void k_na_clear(NoAllocScratch *sc, int n, int ncell) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncell; i += stride)
    sc->cell_head[i] = 0xffffffffu;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    sc->parent[i] = (uint32_t)i;
    sc->next[i] = 0xffffffffu;
  }
  if (blockIdx.x == 0 && threadIdx.x < 4) sc->flags[threadIdx.x] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->ctr = Counters{};
}

template <class PT>
__device__ __forceinline__ int na_cell(const NaGrid &g, const PT *pos, int i, int c[3]) {
  for (int a = 0; a < 3; a++) {
    const double x = (double)pos[3 * i + a];
    if (!(x >= g.rmin[a] && x <= g.rmax[a])) return -1;
    int k = (int)floor(__ddiv_rn(__dsub_rn(x, g.rmin[a]), g.lc));
    c[a] = k < 0 ? 0 : (k >= g.nc[a] ? g.nc[a] - 1 : k);
  }
  return (c[2] * g.nc[1] + c[1]) * g.nc[0] + c[0];
}

template <class PT>
__global__ void k_na_bin(NoAllocScratch *sc, const PT *pos, int n, NaGrid g) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c[3];
    const int cell = na_cell(g, pos, i, c);
    if (cell < 0) {
      atomicAdd(&sc->flags[0], 1u);
      continue;
    }
    sc->next[i] = atomicExch(&sc->cell_head[cell], (uint32_t)i);
  }
}

// The reference's pair predicate in double (FOF.c:351-357), dx in the
// storage precision.
template <class PT>
__device__ __forceinline__ bool na_linked(const PT *pos, int i, int j, double linksq) {
  double d[3];
  for (int a = 0; a < 3; a++) {
    if constexpr (sizeof(PT) == 4) d[a] = (double)__fsub_rn(pos[3 * i + a], pos[3 * j + a]);
    else d[a] = __dsub_rn(pos[3 * i + a], pos[3 * j + a]);
  }
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])),
                              __dmul_rn(d[2], d[2]));
  return !(d2 > linksq);
}

template <class PT>
__global__ void k_na_befriend(NoAllocScratch *sc, const PT *pos, int n, NaGrid g) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c[3];
    if (na_cell(g, pos, i, c) < 0) continue;
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
          if (x < 0 || y < 0 || z < 0 || x >= g.nc[0] || y >= g.nc[1] || z >= g.nc[2]) continue;
          for (uint32_t j = sc->cell_head[(z * g.nc[1] + y) * g.nc[0] + x]; j != 0xffffffffu;
               j = sc->next[j]) {
            if ((int)j <= i) continue;  // each unordered pair once
            if (uf_find(sc->parent, (uint32_t)i) == uf_find(sc->parent, j)) continue;
            if (na_linked(pos, i, (int)j, g.linksq)) uf_union(sc->parent, (uint32_t)i, j, &sc->ctr);
          }
        }
  }
}

// label = root = lowest index of the group (hook-to-min union-find)
__global__ void k_na_label(NoAllocScratch *sc, int n, uint32_t *label) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    label[i] = uf_find(sc->parent, (uint32_t)i);
}

}  // namespace
}  // namespace cmh

extern "C" cmh_status cmh_fof_labels_noalloc(const cmh_fof_params *params, const void *pos,
                                             int32_t pos_dtype, int64_t n, uint32_t *label,
                                             void *stream) {
  using namespace cmh;
  try {
    if (!params || (n > 0 && (!pos || !label)) || n < 0)
      fail(CMH_ERR_INVALID_ARGUMENT, "params, device positions and labels are required");
    if (pos_dtype != CMH_FLOAT32 && pos_dtype != CMH_FLOAT64)
      fail(CMH_ERR_INVALID_ARGUMENT, "unknown position dtype");
    if (params->periodic || params->varlink)
      fail(CMH_ERR_INVALID_ARGUMENT, "the allocation-free variant is non-periodic, constant l");
    if (!(params->linklength > 0) || !(params->boundary >= 0))
      fail(CMH_ERR_INVALID_ARGUMENT, "Linklength must be > 0 and Boundarysize >= 0");
    if (n > kMaxParticles)
      fail(CMH_ERR_CAPACITY, "the allocation-free variant takes at most 65536 particles");
    if (n == 0) return CMH_OK;
    int dev = 0;
    CMH_CUDA(cudaGetDevice(&dev));
    NoAllocScratch *sc = scratch_on(dev);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    NaGrid g{};
    double ext[3];
    for (int a = 0; a < 3; a++) {
      g.rmin[a] = params->lo[a] - params->boundary;
      g.rmax[a] = params->hi[a] + params->boundary;
      ext[a] = g.rmax[a] - g.rmin[a];
      if (!(ext[a] > 0) || !std::isfinite(ext[a]))
        fail(CMH_ERR_INVALID_ARGUMENT, "empty or unbounded domain");
    }
    g.linksq = params->linklength * params->linklength;
    // Cells no smaller than the linking length (so the 27-cell scan sees
    // every linked pair), and at least as large as the side that spreads the
    // padded domain over kMaxCells cells.  Counts are formed in double and
    // checked before any conversion to int.
    g.lc = std::max(params->linklength, std::cbrt(ext[0] * ext[1] * ext[2] / (double)kMaxCells));
    double cells[3] = {0, 0, 0};
    for (int it = 0;; it++) {
      double total = 1.0;
      for (int a = 0; a < 3; a++) {
        cells[a] = std::floor(ext[a] / g.lc) + 1.0;
        total *= cells[a];
      }
      if (total <= (double)kMaxCells) break;
      if (it >= 64 || !std::isfinite(g.lc))
        fail(CMH_ERR_INVALID_ARGUMENT, "no cell grid of at most 2^18 cells covers the domain");
      g.lc *= 1.25;
    }
    for (int a = 0; a < 3; a++) g.nc[a] = (int)cells[a];  // each <= kMaxCells
    int64_t ncell = (int64_t)g.nc[0] * g.nc[1] * g.nc[2];
    const int ni = (int)n;
    const unsigned grid = grid_for(ncell > n ? ncell : n, kThreads, 4);
    k_na_clear<<<grid, kThreads, 0, s>>>(sc, ni, (int)ncell);
    CMH_LAUNCHED();
    const unsigned gp = grid_for(n, kThreads, 4);
    if (pos_dtype == CMH_FLOAT32) {
      k_na_bin<float><<<gp, kThreads, 0, s>>>(sc, (const float *)pos, ni, g);
      CMH_LAUNCHED();
      k_na_befriend<float><<<gp, kThreads, 0, s>>>(sc, (const float *)pos, ni, g);
      CMH_LAUNCHED();
    } else {
      k_na_bin<double><<<gp, kThreads, 0, s>>>(sc, (const double *)pos, ni, g);
      CMH_LAUNCHED();
      k_na_befriend<double><<<gp, kThreads, 0, s>>>(sc, (const double *)pos, ni, g);
      CMH_LAUNCHED();
    }
    k_na_label<<<gp, kThreads, 0, s>>>(sc, ni, label);
    CMH_LAUNCHED();
    unsigned int flags[4] = {0, 0, 0, 0};
    Counters ctr{};
    CMH_CUDA(cudaMemcpyAsync(flags, sc->flags, sizeof flags, cudaMemcpyDeviceToHost, s));
    CMH_CUDA(cudaMemcpyAsync(&ctr, &sc->ctr, sizeof ctr, cudaMemcpyDeviceToHost, s));
    CMH_CUDA(cudaStreamSynchronize(s));
    if (flags[0]) fail(CMH_ERR_DOMAIN, "particles outside [lo - Boundarysize, hi + Boundarysize]");
    if (ctr.uf_giveups) fail(CMH_ERR_DEVICE_TIMEOUT, "union-find retry loop reached its cap");
    return CMH_OK;
  } catch (const Error &e) {
    set_error(e.msg);
    return e.code;
  }
}
