// The FoF hot path on one B200: ingest + periodic images, cell keys, radix
// sort, fine-cell runs, befriending with a lock-free union-find, and the
// segmented reductions that produce the halo catalog.
//
// Reference: src_v2/FOF.c (FOF, Befriend, Checkhalo, Output_Halos property
// sums) and src_v2/read_data.c:409-424,785-816 (domain filter, ghost wrap).
//
// Cells.  Particles are keyed by a fine cell of side h <= l_min / sqrt(3)
// (with a 2^-20 margin): two particles in the same fine cell are closer than
// the linking length whatever their position inside it, so every occupied
// fine cell is one connected piece and union-find runs over cells, not
// particles.  Fine cells are grouped k^3 to a top cell; the sort key is
// (top cell, fine cell inside it), so a top cell's fine cells are contiguous
// and the befriending step visits the 27-cell top stencil (self + 13
// forward neighbours), exactly the cell loop of FOF.c:96-161 one level up.
//
// Pair predicate.  A pair of particles is linked iff the reference's double
// expression ((dx*dx + dy*dy) + dz*dz) <= Linklength^2 holds (FOF.c:351-357),
// dx being a float subtraction for float positions (MEMORY_MODE).
// CMH_PLAIN_FP64 evaluates exactly that for every pair.  CMH_FP32_RECHECK
// evaluates d2_32 = fma(dz,dz, fma(dy,dy, dx*dx)) in FP32 and re-tests in
// double only when t_lo <= d2_32 <= t_hi.  Band proof, float positions:
//   dx is the same float in both paths.  With u = 2^-24 and D the exact sum
//   of the three (exactly representable in double) squares,
//   |d2_32 - D| <= g3 D (g3 = 3u/(1-3u): each term sees at most three
//   roundings), and the reference's value d2_64 = D (1 + t), |t| <= 2^-52.
//   t_lo = fl32(l2) - 4 ulp, with |fl32(l2) - l2| <= ulp/2 and ulp > u l2,
//   so d2_32 < t_lo gives D < l2 (1 - 3.5u) / (1 - g3) < l2 (1 - 0.4u) and
//   hence d2_64 < l2: linked.  Symmetrically d2_32 > t_hi gives d2_64 > l2.
//   For double positions dx_32 = fl32(dx_64) adds 2u, and the band is 8 ulp.
//   Subnormal squares add at most 3 * 2^-149 in absolute terms, far below
//   the 0.4u l2 margin for any linking length above 1e-15.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "cmh_internal.cuh"
#include "fof_kernels.cuh"
#include "plan.cuh"

namespace cmh {

namespace {

constexpr int kT = 256;              // threads per block for element-wise kernels
constexpr uint32_t kNone = 0xffffffffu;
constexpr uint64_t kM21 = (1ull << 21) - 1;

__constant__ int kFwd[14][3] = {
    {0, 0, 0},                                                   // self
    {1, 0, 0},   {-1, 1, 0}, {0, 1, 0},  {1, 1, 0},              // same z
    {-1, -1, 1}, {0, -1, 1}, {1, -1, 1}, {-1, 0, 1}, {0, 0, 1},  // z + 1
    {1, 0, 1},   {-1, 1, 1}, {0, 1, 1},  {1, 1, 1}};

__device__ __forceinline__ int64_t gtid() {
  return (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ int64_t gstride() { return (int64_t)gridDim.x * blockDim.x; }

template <class T> __device__ __forceinline__ double as_d(T v) { return (double)v; }

// ---------------------------------------------------------------------------
// Ingest: domain filter (read_data.c:409-424) and periodic images.
// ---------------------------------------------------------------------------

template <class PT>
__device__ __forceinline__ bool in_domain(const Geom &g, const double x[3]) {
  bool ok = true;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double lo = g.periodic ? g.lo[a] : g.rmin[a];
    double hi = g.periodic ? g.hi[a] : g.rmax[a];
    ok &= (x[a] >= lo) && (x[a] <= hi);  // NaN is outside
  }
  return ok;
}

// Image shift s in {-1, +1} along axis a: the stored coordinate and whether
// it lies in the shell [lo-b, hi+b] (the reference's read_data.c:792-797
// wrap, with the range check of read_data.c:810-812).
template <class PT>
__device__ __forceinline__ bool image_coord(const Geom &g, double x, int a, int s, double *c) {
  double v = __dadd_rn(x, s > 0 ? g.L[a] : -g.L[a]);
  double st = (double)(PT)v;
  *c = st;
  return st >= g.rmin[a] && st <= g.rmax[a];
}

template <class PT>
__global__ void __launch_bounds__(kT) k_ingest_count(const PT *__restrict__ pos, int64_t n,
                                                     Geom g, uint32_t *__restrict__ keep,
                                                     uint32_t *__restrict__ nimg) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    double x[3] = {as_d(pos[3 * i]), as_d(pos[3 * i + 1]), as_d(pos[3 * i + 2])};
    const bool ok = in_domain<PT>(g, x);
    uint32_t cnt = 0;
    if (ok && g.periodic) {
      int opt[3];
#pragma unroll
      for (int a = 0; a < 3; a++) {
        double c;
        opt[a] = 1 + (int)image_coord<PT>(g, x[a], a, -1, &c) + (int)image_coord<PT>(g, x[a], a, 1, &c);
      }
      cnt = (uint32_t)(opt[0] * opt[1] * opt[2] - 1);
    }
    keep[i] = ok ? 1u : 0u;
    nimg[i] = cnt;
  }
}

template <class PT>
__device__ __forceinline__ void emit_one(const Geom &g, uint32_t p, const double c[3],
                                         uint32_t src, uint64_t *keys, uint32_t *vals,
                                         SPos<PT> *ppos) {
  int gi[3];
#pragma unroll
  for (int a = 0; a < 3; a++) gi[a] = fine_index(c[a], g.rmin[a], g.inv_h, g.G[a]);
  const int k = g.k;
  const uint64_t top = ((uint64_t)(gi[2] / k) * g.T[1] + (gi[1] / k)) * g.T[0] + (gi[0] / k);
  const uint64_t sub = ((uint64_t)(gi[2] % k) * k + (gi[1] % k)) * k + (gi[0] % k);
  keys[p] = top * g.k3 + sub;
  vals[p] = p;
  SPos<PT> s;
  s.x = (PT)c[0];
  s.y = (PT)c[1];
  s.z = (PT)c[2];
  s.src = src;
  ppos[p] = s;
}

// Processing order: kept originals in input order, then the images grouped
// by source particle and shift code (sz+1)*9 + (sy+1)*3 + (sx+1) ascending.
template <class PT>
__global__ void __launch_bounds__(kT) k_ingest_emit(
    const PT *__restrict__ pos, int64_t n, Geom g, const uint32_t *__restrict__ keep,
    const uint32_t *__restrict__ keep_scan, const uint32_t *__restrict__ img_scan,
    const uint32_t *__restrict__ nimg, const uint32_t *__restrict__ nkept_ptr,
    uint64_t *__restrict__ keys, uint32_t *__restrict__ vals, SPos<PT> *__restrict__ ppos) {
  const uint32_t nkept = *nkept_ptr;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    if (!keep[i]) continue;
    double x[3] = {as_d(pos[3 * i]), as_d(pos[3 * i + 1]), as_d(pos[3 * i + 2])};
    emit_one<PT>(g, keep_scan[i], x, (uint32_t)i, keys, vals, ppos);
    if (!g.periodic || nimg[i] == 0) continue;
    uint32_t q = nkept + img_scan[i];
    double cm[3], cp[3];
    bool okm[3], okp[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      okm[a] = image_coord<PT>(g, x[a], a, -1, &cm[a]);
      okp[a] = image_coord<PT>(g, x[a], a, 1, &cp[a]);
    }
    for (int code = 0; code < 27; code++) {
      if (code == 13) continue;
      const int s[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
      double c[3];
      bool ok = true;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        if (s[a] < 0) { ok &= okm[a]; c[a] = cm[a]; }
        else if (s[a] > 0) { ok &= okp[a]; c[a] = cp[a]; }
        else c[a] = x[a];
      }
      if (!ok) continue;
      emit_one<PT>(g, q++, c, (uint32_t)i, keys, vals, ppos);
    }
  }
}

// ---------------------------------------------------------------------------
// Runs of equal fine-cell keys.
// ---------------------------------------------------------------------------

template <class PT>
__global__ void __launch_bounds__(kT) k_gather_flags(const uint64_t *__restrict__ keys,
                                                     const uint32_t *__restrict__ perm,
                                                     const SPos<PT> *__restrict__ ppos,
                                                     SPos<PT> *__restrict__ spos,
                                                     uint32_t *__restrict__ flag, int64_t np) {
  for (int64_t i = gtid(); i < np; i += gstride()) {
    spos[i] = ppos[perm[i]];
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
  }
}

__global__ void __launch_bounds__(kT) k_runs(const uint64_t *__restrict__ keys,
                                             const uint32_t *__restrict__ flag,
                                             const uint32_t *__restrict__ run_scan, int64_t np,
                                             Geom g, uint32_t *__restrict__ run_of,
                                             uint32_t *__restrict__ run_start,
                                             uint64_t *__restrict__ run_g,
                                             const uint32_t *__restrict__ nruns) {
  const uint32_t R = *nruns;
  for (int64_t i = gtid(); i < np; i += gstride()) {
    const uint32_t rid = run_scan[i] + flag[i] - 1u;
    run_of[i] = rid;
    if (flag[i]) {
      run_start[rid] = (uint32_t)i;
      const uint64_t key = keys[i];
      const uint64_t top = key / g.k3, sub = key % g.k3;
      const int k = g.k;
      const uint64_t tx = top % g.T[0], ty = (top / g.T[0]) % g.T[1], tz = top / ((uint64_t)g.T[0] * g.T[1]);
      const uint64_t sx = sub % k, sy = (sub / k) % k, sz = sub / ((uint64_t)k * k);
      const uint64_t gx = tx * k + sx, gy = ty * k + sy, gz = tz * k + sz;
      run_g[rid] = gx | (gy << 21) | (gz << 42);
    }
    if (i == np - 1) run_start[R] = (uint32_t)np;
  }
}

__device__ __forceinline__ uint64_t top_of_run(const Geom &g, uint64_t pg) {
  const int k = g.k;
  const uint64_t gx = pg & kM21, gy = (pg >> 21) & kM21, gz = pg >> 42;
  return ((gz / k) * g.T[1] + gy / k) * g.T[0] + gx / k;
}

__global__ void __launch_bounds__(kT) k_top_ranges(const uint64_t *__restrict__ run_g, Geom g,
                                                   const uint32_t *__restrict__ nruns,
                                                   uint32_t *__restrict__ top_first,
                                                   uint32_t *__restrict__ top_end) {
  const uint32_t R = *nruns;
  for (int64_t r = gtid(); r < R; r += gstride()) {
    const uint64_t t = top_of_run(g, run_g[r]);
    if (r == 0 || top_of_run(g, run_g[r - 1]) != t) top_first[t] = (uint32_t)r;
    if (r == R - 1 || top_of_run(g, run_g[r + 1]) != t) top_end[t] = (uint32_t)(r + 1);
  }
}

__global__ void __launch_bounds__(kT) k_dense_flags(const uint64_t *__restrict__ run_g, Geom g,
                                                    const uint32_t *__restrict__ nruns,
                                                    const uint32_t *__restrict__ top_first,
                                                    const uint32_t *__restrict__ top_end,
                                                    uint32_t dense_min,
                                                    uint32_t *__restrict__ flag) {
  const uint32_t R = *nruns;
  for (int64_t r = gtid(); r < R; r += gstride()) {
    const uint64_t t = top_of_run(g, run_g[r]);
    flag[r] = (top_first[t] == (uint32_t)r && top_end[t] - top_first[t] > dense_min) ? 1u : 0u;
  }
}

__global__ void __launch_bounds__(kT) k_dense_maps(const uint64_t *__restrict__ run_g, Geom g,
                                                   const uint32_t *__restrict__ nruns,
                                                   const uint32_t *__restrict__ top_first,
                                                   const uint32_t *__restrict__ top_end,
                                                   const uint32_t *__restrict__ dflag,
                                                   const uint32_t *__restrict__ dscan,
                                                   uint32_t dense_min,
                                                   uint32_t *__restrict__ top_slot,
                                                   uint2 *__restrict__ dense_range,
                                                   int32_t *__restrict__ maps) {
  const uint32_t R = *nruns;
  const int k = g.k;
  for (int64_t r = gtid(); r < R; r += gstride()) {
    const uint64_t pg = run_g[r];
    const uint64_t t = top_of_run(g, pg);
    const uint32_t f = top_first[t];
    if (top_end[t] - f <= dense_min) continue;
    const uint32_t slot = dscan[f];  // the first run of the cell carries the slot
    if (dflag[r]) {
      top_slot[t] = slot;
      dense_range[slot] = make_uint2(f, top_end[t]);
    }
    const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
    const uint64_t sub = ((uint64_t)(gz % k) * k + (gy % k)) * k + (gx % k);
    maps[(uint64_t)slot * g.k3 + sub] = (int32_t)r;
  }
}

__global__ void __launch_bounds__(kT) k_iota(uint32_t *__restrict__ a,
                                             const uint32_t *__restrict__ nruns) {
  const uint32_t R = *nruns;
  for (int64_t r = gtid(); r < R; r += gstride()) a[r] = (uint32_t)r;
}

// ---------------------------------------------------------------------------
// Befriending.
// ---------------------------------------------------------------------------

// The reference's pair predicate (FOF.c:351-357), FP64 or FP32 + band recheck.
template <class PT, bool FP32>
__device__ __forceinline__ bool linked(const SPos<PT> &p, const SPos<PT> &q, const Geom &g,
                                       unsigned long long &rechecks) {
  double dx, dy, dz;
  if constexpr (sizeof(PT) == 4) {
    const float fx = __fsub_rn(p.x, q.x), fy = __fsub_rn(p.y, q.y), fz = __fsub_rn(p.z, q.z);
    if constexpr (FP32) {
      const float d2 = __fmaf_rn(fz, fz, __fmaf_rn(fy, fy, __fmul_rn(fx, fx)));
      if (d2 < g.t_lo) return true;
      if (d2 > g.t_hi) return false;
      rechecks++;
    }
    dx = (double)fx;
    dy = (double)fy;
    dz = (double)fz;
  } else {
    dx = __dsub_rn(p.x, q.x);
    dy = __dsub_rn(p.y, q.y);
    dz = __dsub_rn(p.z, q.z);
    if constexpr (FP32) {
      const float fx = __double2float_rn(dx), fy = __double2float_rn(dy),
                  fz = __double2float_rn(dz);
      const float d2 = __fmaf_rn(fz, fz, __fmaf_rn(fy, fy, __fmul_rn(fx, fx)));
      if (d2 < g.t_lo) return true;
      if (d2 > g.t_hi) return false;
      rechecks++;
    }
  }
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return !(d2 > g.linksq);
}

// Squared distance from a point to the box of fine cell (cx, cy, cz).
__device__ __forceinline__ double box_dist2(const Geom &g, double x, double y, double z, int cx,
                                            int cy, int cz) {
  const double bx = __dadd_rn(g.rmin[0], __dmul_rn((double)cx, g.h));
  const double by = __dadd_rn(g.rmin[1], __dmul_rn((double)cy, g.h));
  const double bz = __dadd_rn(g.rmin[2], __dmul_rn((double)cz, g.h));
  const double ex = fmax(0.0, fmax(bx - x, x - (bx + g.h)));
  const double ey = fmax(0.0, fmax(by - y, y - (by + g.h)));
  const double ez = fmax(0.0, fmax(bz - z, z - (bz + g.h)));
  return ex * ex + ey * ey + ez * ez;
}

// Per-thread tallies of the befriending kernel, flushed once per warp.
struct BfStats {
  unsigned long long tests = 0, rechecks = 0, cand = 0, skips = 0, unions = 0, steps = 0;
  unsigned long long scan = 0, window = 0;
};

// Whether any particle of fine cell a (particles [sa, ea)) is linked to any
// particle of fine cell b (fine coordinates bx, by, bz).  Particles of a
// farther than the linking length from b's box are skipped.  Every 16
// particles of a, `apart()` is asked whether a and b are still in different
// components (another thread may have joined them meanwhile); if not, the
// search stops and reports no link, which is then harmless.
template <class PT, bool FP32, class Apart>
__device__ __forceinline__ bool cells_linked(const Geom &g, uint32_t b, int bx, int by, int bz,
                                             uint32_t sa, uint32_t ea,
                                             const uint32_t *__restrict__ run_start,
                                             const SPos<PT> *__restrict__ spos, BfStats &st,
                                             Apart apart) {
  const uint32_t sb = __ldg(run_start + b), eb = __ldg(run_start + b + 1);
  for (uint32_t i = sa; i < ea; i++) {
    if (((i - sa) & 15) == 15 && !apart()) return false;
    const SPos<PT> p = spos[i];
    if (box_dist2(g, (double)p.x, (double)p.y, (double)p.z, bx, by, bz) > g.prune_sq) continue;
    for (uint32_t j = sb; j < eb; j++) {
      st.tests++;
      if (linked<PT, FP32>(p, spos[j], g, st.rechecks)) return true;
    }
  }
  return false;
}

// Link fine cells a and b if any pair of their particles is linked.  The
// cells are internally connected, so one linked pair joins them entirely.
// `ra` caches a root of a's component: it may be stale (a root that was hooked
// since), but it stays in a's component, so "b reaches ra" still proves that
// a and b are already joined.
template <class PT, bool FP32>
__device__ __forceinline__ void try_link(const Geom &g, uint32_t a, uint32_t &ra, uint32_t b,
                                         int bx, int by, int bz, uint32_t sa, uint32_t ea,
                                         const uint32_t *__restrict__ run_start,
                                         const SPos<PT> *__restrict__ spos, uint32_t *parent,
                                         Counters *ctr, BfStats &st) {
  st.cand++;
  const uint32_t pb = __ldcg(parent + b);
  st.steps++;
  if (pb == ra) { st.skips++; return; }
  const uint32_t rb = (pb == b) ? b : uf_find_n(parent, pb, st.steps);
  if (rb == ra) { st.skips++; return; }
  ra = uf_find_n(parent, ra, st.steps);
  if (rb == ra) { st.skips++; return; }
  auto apart = [&]() {
    return uf_find_n(parent, a, st.steps) != uf_find_n(parent, b, st.steps);
  };
  if (cells_linked<PT, FP32>(g, b, bx, by, bz, sa, ea, run_start, spos, st, apart)) {
    uf_union(parent, ra, rb, ctr);
    st.unions++;
    ra = uf_find_n(parent, ra, st.steps);
  }
}

// Union-find in shared memory over the fine cells of one top cell (local
// indices), same hook-to-min rule as the global one.
__device__ __forceinline__ uint32_t lfind(volatile uint32_t *lp, uint32_t x) {
  while (true) {
    const uint32_t p = lp[x];
    if (p == x) return x;
    const uint32_t gp = lp[p];
    if (gp == p) return p;
    lp[x] = gp;
    x = gp;
  }
}

__device__ __forceinline__ void lunion(uint32_t *lp, uint32_t a, uint32_t b, Counters *ctr) {
  for (int it = 0; it < kUnionCap; it++) {
    a = lfind(lp, a);
    b = lfind(lp, b);
    if (a == b) return;
    if (a < b) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    const uint32_t old = atomicCAS(lp + a, a, b);
    if (old == a) return;
    a = old;
  }
  atomicAdd(&ctr->uf_giveups, 1u);
}

// Dense top cells, one CTA each: the fine-cell pairs inside the top cell are
// joined with a shared-memory union-find (neighbours found through the top
// cell's fine-cell map), near pairs before far ones; then every fine cell's
// global parent is set to its local root.  Links that cross the top cell's
// faces are left to the global passes.
template <class PT, bool FP32>
__global__ void __launch_bounds__(128) k_befriend_dense(
    Geom g, const uint32_t *__restrict__ run_start, const uint64_t *__restrict__ run_g,
    const uint2 *__restrict__ dense_range, const uint32_t *__restrict__ ndense, uint32_t *next,
    const int32_t *__restrict__ maps, const SPos<PT> *__restrict__ spos, uint32_t *parent,
    Counters *ctr) {
  extern __shared__ uint32_t lpar[];
  __shared__ uint32_t s_slot;
  const uint32_t nd = *ndense;
  const int k = g.k, W = g.W;
  BfStats st;
  while (true) {
    // top cells are taken from an atomic counter: their sizes differ widely
    if (threadIdx.x == 0) s_slot = atomicAdd(next, 1u);
    __syncthreads();
    const uint32_t slot = s_slot;
    __syncthreads();
    if (slot >= nd) break;
    const uint2 fr = dense_range[slot];
    const uint32_t f = fr.x, n = fr.y - fr.x;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) lpar[i] = i;
    __syncthreads();
    const int32_t *map = maps + (uint64_t)slot * g.k3;
    for (int pass = 0; pass < 2; pass++) {
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t a = f + i;
        const uint64_t pg = run_g[a];
        const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
        const int sx = gx % k, sy = gy % k, sz = gz % k;
        const uint32_t sa = run_start[a], ea = run_start[a + 1];
        for (int dz = 0; dz <= W; dz++)
          for (int dy = -W; dy <= W; dy++)
            for (int dx = -W; dx <= W; dx++) {
              if (dz == 0 && (dy < 0 || (dy == 0 && dx <= 0))) continue;  // forward only
              const int cheb = max(abs(dx), max(abs(dy), dz));
              if ((pass == 0) != (cheb <= 1)) continue;
              const int tx = sx + dx, ty = sy + dy, tz = sz + dz;
              if (tx < 0 || ty < 0 || tx >= k || ty >= k || tz >= k) continue;
              const int32_t r = map[(tz * k + ty) * k + tx];
              if (r < 0) continue;
              st.cand++;
              const uint32_t lj = (uint32_t)r - f;
              const uint32_t ri = lfind(lpar, i), rj = lfind(lpar, lj);
              if (ri == rj) {
                st.skips++;
                continue;
              }
              auto apart = [&]() { return lfind(lpar, i) != lfind(lpar, lj); };
              if (cells_linked<PT, FP32>(g, (uint32_t)r, gx + dx, gy + dy, gz + dz, sa, ea,
                                         run_start, spos, st, apart)) {
                lunion(lpar, ri, rj, ctr);
                st.unions++;
              }
            }
      }
      __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) parent[f + i] = f + lfind(lpar, i);
    __syncthreads();
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    st.tests += __shfl_down_sync(0xffffffffu, st.tests, d);
    st.rechecks += __shfl_down_sync(0xffffffffu, st.rechecks, d);
    st.cand += __shfl_down_sync(0xffffffffu, st.cand, d);
    st.skips += __shfl_down_sync(0xffffffffu, st.skips, d);
    st.unions += __shfl_down_sync(0xffffffffu, st.unions, d);
  }
  if ((threadIdx.x & 31) == 0) {
    if (st.tests) atomicAdd(&ctr->pair_tests, st.tests);
    if (st.rechecks) atomicAdd(&ctr->rechecks, st.rechecks);
    if (st.cand) atomicAdd(&ctr->cand_pairs, st.cand);
    if (st.skips) atomicAdd(&ctr->root_skips, st.skips);
    if (st.unions) atomicAdd(&ctr->unions, st.unions);
  }
}

// Whether fine cell a's neighbour top cell in direction (ox, oy, oz) lies
// within W fine cells of a (s = a's fine coordinates inside its top cell).
__device__ __forceinline__ bool reaches(int s, int o, int k, int W) {
  return o == 0 || (o > 0 ? s >= k - W : s <= W - 1);
}

// Candidates of fine cell a are the fine cells b > a (key order, so each
// unordered pair is visited once) within W fine cells on every axis; they
// live in a's top cell (after a) and the 13 forward top cells.
//
// Fast path, one thread per fine cell: the 14 top-cell ranges are loaded at
// once; when no range holds more than kSimple candidate cells (the common
// case away from clumps), the first of each is loaded at once too and the
// cell is finished in two L2 round trips.  Other cells are queued for the
// warp path below.
constexpr uint32_t kSimple = 2;

template <class PT, bool FP32>
__global__ void __launch_bounds__(kT, 5) k_befriend_simple(
    Geom g, const uint32_t *__restrict__ run_start, const uint64_t *__restrict__ run_g,
    const uint32_t *__restrict__ nruns, const uint32_t *__restrict__ top_first,
    const uint32_t *__restrict__ top_end, uint32_t dense_min,
    const SPos<PT> *__restrict__ spos, uint32_t *parent, uint32_t *__restrict__ queue,
    uint32_t *qcount, Counters *ctr) {
  const uint32_t R = *nruns;
  const int k = g.k, W = g.W;
  const int lane = threadIdx.x & 31;
  BfStats st;
  for (int64_t ai = gtid(); ai < R; ai += gstride()) {
    const uint32_t a = (uint32_t)ai;
    const uint64_t pg = run_g[a];
    const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
    const int tx = gx / k, ty = gy / k, tz = gz / k;
    const int sx = gx - tx * k, sy = gy - ty * k, sz = gz - tz * k;
    uint32_t R0[14], NN[14];
#pragma unroll
    for (int nb = 0; nb < 14; nb++) {
      const int ux = tx + kFwd[nb][0], uy = ty + kFwd[nb][1], uz = tz + kFwd[nb][2];
      // a top cell more than W fine cells away from a is skipped without a load
      const bool in = !(ux < 0 || uy < 0 || ux >= g.T[0] || uy >= g.T[1] || uz >= g.T[2]) &&
                      reaches(sx, kFwd[nb][0], k, W) && reaches(sy, kFwd[nb][1], k, W) &&
                      reaches(sz, kFwd[nb][2], k, W);
      const uint64_t tb = in ? ((uint64_t)uz * g.T[1] + uy) * g.T[0] + ux : 0;
      const uint32_t f = in ? top_first[tb] : 0u, e = in ? top_end[tb] : 0u;
      R0[nb] = nb == 0 ? a + 1 : f;
      NN[nb] = e > R0[nb] ? e - R0[nb] : 0u;
      // pairs inside a dense top cell are joined by k_befriend_dense
      if (nb == 0 && e - f > dense_min) NN[nb] = 0u;
    }
    bool simple = true;
#pragma unroll
    for (int nb = 0; nb < 14; nb++) simple &= NN[nb] <= kSimple;
    const unsigned active = __activemask();
    const unsigned qmask = __ballot_sync(active, !simple);
    if (qmask) {
      const int leader = __ffs(qmask) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(qcount, (uint32_t)__popc(qmask));
      base = __shfl_sync(active, base, leader);
      if (!simple) queue[base + __popc(qmask & ((1u << lane) - 1u))] = a;
    }
    if (!simple) continue;
    uint64_t Q[14];
#pragma unroll
    for (int nb = 0; nb < 14; nb++) Q[nb] = NN[nb] ? run_g[R0[nb]] : 0ull;
    uint32_t ra = 0xffffffffu, sa = 0, ea = 0;
#pragma unroll
    for (int nb = 0; nb < 14; nb++) {
      for (uint32_t q = 0; q < NN[nb]; q++) {
        const uint64_t qg = q == 0 ? Q[nb] : run_g[R0[nb] + q];
        const int bx = (int)(qg & kM21), by = (int)((qg >> 21) & kM21), bz = (int)(qg >> 42);
        st.scan++;
        if (max(abs(bx - gx), max(abs(by - gy), abs(bz - gz))) > W) continue;
        if (ra == 0xffffffffu) {
          ra = __ldcg(parent + a);
          sa = run_start[a];
          ea = run_start[a + 1];
        }
        try_link<PT, FP32>(g, a, ra, R0[nb] + q, bx, by, bz, sa, ea, run_start, spos, parent,
                           ctr, st);
      }
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    st.tests += __shfl_down_sync(0xffffffffu, st.tests, d);
    st.rechecks += __shfl_down_sync(0xffffffffu, st.rechecks, d);
    st.cand += __shfl_down_sync(0xffffffffu, st.cand, d);
    st.skips += __shfl_down_sync(0xffffffffu, st.skips, d);
    st.unions += __shfl_down_sync(0xffffffffu, st.unions, d);
    st.steps += __shfl_down_sync(0xffffffffu, st.steps, d);
    st.scan += __shfl_down_sync(0xffffffffu, st.scan, d);
  }
  if (lane == 0) {
    if (st.tests) atomicAdd(&ctr->pair_tests, st.tests);
    if (st.rechecks) atomicAdd(&ctr->rechecks, st.rechecks);
    if (st.cand) atomicAdd(&ctr->cand_pairs, st.cand);
    if (st.skips) atomicAdd(&ctr->root_skips, st.skips);
    if (st.unions) atomicAdd(&ctr->unions, st.unions);
    if (st.steps) atomicAdd(&ctr->find_steps, st.steps);
    if (st.scan) atomicAdd(&ctr->scan_iters, st.scan);
  }
}

// Warp path, one warp per queued fine cell a.  Lanes 0..13 fetch the 14
// top-cell ranges at once; the candidate slots of all 14 (fine cells of small
// top cells, map slots of the window in dense ones) are then flattened and
// taken 32 at a time, so a cell costs a few L2 round trips instead of one per
// slot.  Warps take cells from `next` (an atomic counter) as they finish, so
// a few expensive cells do not hold back a whole static share.  PHASE 0
// visits the candidates within one fine cell, PHASE 1 the farther ones, so
// that a dense neighbourhood is joined (and compressed) before its far pairs
// are tried and most of those become root skips.
template <class PT, bool FP32, int PHASE>
__global__ void __launch_bounds__(kT) k_befriend(
    Geom g, const uint32_t *__restrict__ run_start, const uint64_t *__restrict__ run_g,
    const uint32_t *__restrict__ queue, const uint32_t *__restrict__ qcount, uint32_t *next,
    const uint32_t *__restrict__ top_first, const uint32_t *__restrict__ top_end,
    const uint32_t *__restrict__ top_slot, const int32_t *__restrict__ maps, uint32_t dense_min,
    const SPos<PT> *__restrict__ spos, uint32_t *parent, Counters *ctr) {
  const uint32_t NQ = *qcount;
  const int k = g.k, W = g.W;
  const int lane = threadIdx.x & 31;
  BfStats st;
  while (true) {
    uint32_t qi = 0;
    if (lane == 0) qi = atomicAdd(next, 1u);
    qi = __shfl_sync(0xffffffffu, qi, 0);
    if (qi >= NQ) break;
    const uint32_t a = queue[qi];
    const uint64_t pg = run_g[a];
    const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
    const int tx = gx / k, ty = gy / k, tz = gz / k;
    const uint32_t sa = run_start[a], ea = run_start[a + 1];
    uint32_t ra = __ldcg(parent + a);
    const int sx = gx - tx * k, sy = gy - ty * k, sz = gz - tz * k;
    // lane l < 14 describes neighbour top cell l
    uint32_t r0 = 0, nsparse = 0, nslots = 0, mapbase = 0;
    int x0 = 0, y0 = 0, z0 = 0, nx = 1, ny = 1, ox = 0, oy = 0, oz = 0;
    if (lane < 14) {
      const int ux = tx + kFwd[lane][0], uy = ty + kFwd[lane][1], uz = tz + kFwd[lane][2];
      if (!(ux < 0 || uy < 0 || ux >= g.T[0] || uy >= g.T[1] || uz >= g.T[2]) &&
          reaches(sx, kFwd[lane][0], k, W) && reaches(sy, kFwd[lane][1], k, W) &&
          reaches(sz, kFwd[lane][2], k, W)) {
        const uint64_t tb = ((uint64_t)uz * g.T[1] + uy) * g.T[0] + ux;
        const uint32_t f = top_first[tb], e = top_end[tb];
        r0 = lane == 0 ? a + 1 : f;
        // pairs inside a dense top cell are joined by k_befriend_dense
        if (lane == 0 && e - f > dense_min) r0 = e;
        if (r0 < e) {
          if (e - f <= dense_min) {
            nsparse = e - r0;
          } else {
            x0 = max(gx - W, ux * k);
            const int x1 = min(gx + W, ux * k + k - 1);
            y0 = max(gy - W, uy * k);
            const int y1 = min(gy + W, uy * k + k - 1);
            // in a's own top cell only rows at or after a's hold cells b > a
            z0 = max(lane == 0 ? gz : gz - W, uz * k);
            const int z1 = min(gz + W, uz * k + k - 1);
            if (x1 >= x0 && y1 >= y0 && z1 >= z0) {
              nx = x1 - x0 + 1;
              ny = y1 - y0 + 1;
              nslots = (uint32_t)(nx * ny * (z1 - z0 + 1));
              mapbase = top_slot[tb];
              ox = ux * k;
              oy = uy * k;
              oz = uz * k;
            }
          }
        }
      }
    }
    const uint32_t cnt = nsparse + nslots;
    uint32_t incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t excl = incl - cnt;
    for (uint32_t j0 = 0; j0 < total; j0 += 32) {
      const uint32_t j = j0 + lane;
      // the neighbour top cell l whose items hold j
      int l = 0;
#pragma unroll
      for (int q = 1; q < 14; q++)
        if (j >= __shfl_sync(0xffffffffu, excl, q)) l = q;
      const uint32_t l_excl = __shfl_sync(0xffffffffu, excl, l);
      const uint32_t l_r0 = __shfl_sync(0xffffffffu, r0, l);
      const uint32_t l_ns = __shfl_sync(0xffffffffu, nsparse, l);
      const int l_x0 = __shfl_sync(0xffffffffu, x0, l), l_y0 = __shfl_sync(0xffffffffu, y0, l),
                l_z0 = __shfl_sync(0xffffffffu, z0, l), l_nx = __shfl_sync(0xffffffffu, nx, l),
                l_ny = __shfl_sync(0xffffffffu, ny, l), l_ox = __shfl_sync(0xffffffffu, ox, l),
                l_oy = __shfl_sync(0xffffffffu, oy, l), l_oz = __shfl_sync(0xffffffffu, oz, l);
      const uint32_t l_map = __shfl_sync(0xffffffffu, mapbase, l);
      if (j >= total) continue;
      const uint32_t off = j - l_excl;
      uint32_t r;
      int bx, by, bz;
      if (off < l_ns) {
        st.scan++;
        r = l_r0 + off;
        const uint64_t qg = run_g[r];
        bx = (int)(qg & kM21);
        by = (int)((qg >> 21) & kM21);
        bz = (int)(qg >> 42);
        if (max(abs(bx - gx), max(abs(by - gy), abs(bz - gz))) > W) continue;
      } else {
        st.window++;
        const uint32_t sl = off - l_ns;
        bx = l_x0 + (int)(sl % (uint32_t)l_nx);
        by = l_y0 + (int)((sl / (uint32_t)l_nx) % (uint32_t)l_ny);
        bz = l_z0 + (int)(sl / (uint32_t)(l_nx * l_ny));
        const int32_t rr =
            maps[(uint64_t)l_map * g.k3 + (uint64_t)(((bz - l_oz) * k + (by - l_oy)) * k + (bx - l_ox))];
        if (rr < 0 || (uint32_t)rr < l_r0) continue;
        r = (uint32_t)rr;
      }
      const int cheb = max(abs(bx - gx), max(abs(by - gy), abs(bz - gz)));
      if ((PHASE == 0 && cheb > 1) || (PHASE == 1 && cheb <= 1)) continue;
      try_link<PT, FP32>(g, a, ra, r, bx, by, bz, sa, ea, run_start, spos, parent, ctr, st);
    }
  }
  // one atomic per warp for the counters
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    st.tests += __shfl_down_sync(0xffffffffu, st.tests, d);
    st.rechecks += __shfl_down_sync(0xffffffffu, st.rechecks, d);
    st.cand += __shfl_down_sync(0xffffffffu, st.cand, d);
    st.skips += __shfl_down_sync(0xffffffffu, st.skips, d);
    st.unions += __shfl_down_sync(0xffffffffu, st.unions, d);
    st.steps += __shfl_down_sync(0xffffffffu, st.steps, d);
    st.scan += __shfl_down_sync(0xffffffffu, st.scan, d);
    st.window += __shfl_down_sync(0xffffffffu, st.window, d);
  }
  if ((threadIdx.x & 31) == 0) {
    if (st.tests) atomicAdd(&ctr->pair_tests, st.tests);
    if (st.rechecks) atomicAdd(&ctr->rechecks, st.rechecks);
    if (st.cand) atomicAdd(&ctr->cand_pairs, st.cand);
    if (st.skips) atomicAdd(&ctr->root_skips, st.skips);
    if (st.unions) atomicAdd(&ctr->unions, st.unions);
    if (st.steps) atomicAdd(&ctr->find_steps, st.steps);
    if (st.scan) atomicAdd(&ctr->scan_iters, st.scan);
    if (st.window) atomicAdd(&ctr->window_iters, st.window);
  }
}

__global__ void __launch_bounds__(kT) k_compress(uint32_t *parent,
                                                 const uint32_t *__restrict__ nruns) {
  const uint32_t R = *nruns;
  for (int64_t r = gtid(); r < R; r += gstride()) parent[r] = uf_find(parent, (uint32_t)r);
}

// ---------------------------------------------------------------------------
// Segmented reductions over cell-ordered particles.
// ---------------------------------------------------------------------------

// Lanes of a warp holding the same key in adjacent lanes form a segment; the
// segment's first lane receives the segment's sum of v (and min of m).
template <int NV>
__device__ __forceinline__ bool warp_segments(uint32_t key, double (&v)[NV]) {
  const int lane = threadIdx.x & 31;
  const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool head = lane == 0 || prev != key;
  const uint32_t heads = __ballot_sync(0xffffffffu, head);
  const uint32_t seg = __popc(heads & ((2u << lane) - 1u));  // 1-based segment id
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t oseg = __shfl_down_sync(0xffffffffu, seg, d);
    const bool take = (lane + d < 32) && oseg == seg;
#pragma unroll
    for (int c = 0; c < NV; c++) {
      const double t = __shfl_down_sync(0xffffffffu, v[c], d);
      if (take) v[c] += t;
    }
  }
  return head;
}

__device__ __forceinline__ bool warp_segments_count_min(uint32_t key, uint32_t &cnt,
                                                        uint32_t &mn) {
  const int lane = threadIdx.x & 31;
  const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool head = lane == 0 || prev != key;
  const uint32_t heads = __ballot_sync(0xffffffffu, head);
  const uint32_t seg = __popc(heads & ((2u << lane) - 1u));
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t oseg = __shfl_down_sync(0xffffffffu, seg, d);
    const uint32_t oc = __shfl_down_sync(0xffffffffu, cnt, d);
    const uint32_t om = __shfl_down_sync(0xffffffffu, mn, d);
    if ((lane + d < 32) && oseg == seg) {
      cnt += oc;
      mn = min(mn, om);
    }
  }
  return head;
}

// Group size and head (lowest processing index) per root cell.
__global__ void __launch_bounds__(kT) k_group_count(const uint32_t *__restrict__ run_of,
                                                    const uint32_t *__restrict__ parent,
                                                    const uint32_t *__restrict__ perm, int64_t np,
                                                    uint32_t *__restrict__ count,
                                                    uint32_t *__restrict__ head) {
  const int64_t n_iter = (np + 31) / 32 * 32;
  for (int64_t i = gtid(); i < n_iter; i += gstride()) {
    const bool valid = i < np;
    const uint32_t root = valid ? parent[run_of[i]] : kNone;
    uint32_t c = valid ? 1u : 0u;
    uint32_t m = valid ? perm[i] : kNone;
    const bool h = warp_segments_count_min(root, c, m);
    if (valid && h) {
      atomicAdd(count + root, c);
      atomicMin(head + root, m);
    }
  }
}

__global__ void __launch_bounds__(kT) k_cand_flags(const uint32_t *__restrict__ parent,
                                                   const uint32_t *__restrict__ count,
                                                   const uint32_t *__restrict__ nruns,
                                                   double nphalomin, uint32_t *__restrict__ flag,
                                                   unsigned long long *ngroups) {
  const uint32_t R = *nruns;
  unsigned long long roots = 0;
  for (int64_t r = gtid(); r < R; r += gstride()) {
    const bool root = parent[r] == (uint32_t)r;
    roots += root;
    flag[r] = (root && !((double)count[r] < nphalomin)) ? 1u : 0u;  // FOF.c:202
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) roots += __shfl_down_sync(0xffffffffu, roots, d);
  if ((threadIdx.x & 31) == 0 && roots) atomicAdd(ngroups, roots);
}

__global__ void __launch_bounds__(kT) k_cand_list(const uint32_t *__restrict__ flag,
                                                  const uint32_t *__restrict__ scan,
                                                  const uint32_t *__restrict__ nruns,
                                                  uint32_t *__restrict__ cand_of_root,
                                                  uint32_t *__restrict__ cand_root) {
  const uint32_t R = *nruns;
  for (int64_t r = gtid(); r < R; r += gstride()) {
    if (!flag[r]) continue;
    cand_of_root[r] = scan[r];
    cand_root[scan[r]] = (uint32_t)r;
  }
}

// Property sums per candidate halo, in double as Output_Halos does
// (FOF.c:806-832): 6 first moments, then 6 position and 6 velocity second
// moments when INERTIA / DISPERSION are asked for.
template <class PT, class VT, int NS>
__global__ void __launch_bounds__(kT) k_group_sums(
    const uint32_t *__restrict__ run_of, const uint32_t *__restrict__ parent,
    const uint32_t *__restrict__ cand_of_root, const SPos<PT> *__restrict__ spos,
    const VT *__restrict__ vel, int64_t np, Geom g, double *__restrict__ sums,
    uint32_t *__restrict__ warn) {
  const int64_t n_iter = (np + 31) / 32 * 32;
  for (int64_t i = gtid(); i < n_iter; i += gstride()) {
    uint32_t ci = kNone;
    double v[NS];
#pragma unroll
    for (int c = 0; c < NS; c++) v[c] = 0.0;
    if (i < np) {
      ci = cand_of_root[parent[run_of[i]]];
      if (ci != kNone) {
        const SPos<PT> p = spos[i];
        const double x = (double)p.x, y = (double)p.y, z = (double)p.z;
        const double vx = (double)vel[3 * (uint64_t)p.src], vy = (double)vel[3 * (uint64_t)p.src + 1],
                     vz = (double)vel[3 * (uint64_t)p.src + 2];
        v[0] = x; v[1] = y; v[2] = z; v[3] = vx; v[4] = vy; v[5] = vz;
        if constexpr (NS >= 12) {
          if (g.props & 1) {
            v[6] = __dmul_rn(x, x); v[7] = __dmul_rn(y, y); v[8] = __dmul_rn(z, z);
            v[9] = __dmul_rn(x, y); v[10] = __dmul_rn(x, z); v[11] = __dmul_rn(y, z);
          }
        }
        if constexpr (NS >= 18) {
          v[12] = __dmul_rn(vx, vx); v[13] = __dmul_rn(vy, vy); v[14] = __dmul_rn(vz, vz);
          v[15] = __dmul_rn(vx, vy); v[16] = __dmul_rn(vx, vz); v[17] = __dmul_rn(vy, vz);
        } else if constexpr (NS >= 12) {
          if (!(g.props & 1)) {
            v[6] = __dmul_rn(vx, vx); v[7] = __dmul_rn(vy, vy); v[8] = __dmul_rn(vz, vz);
            v[9] = __dmul_rn(vx, vy); v[10] = __dmul_rn(vx, vz); v[11] = __dmul_rn(vy, vz);
          }
        }
        // edge warning of Checkhalo (FOF.c:406-422)
        if (x - g.rmin[0] < g.maxlink || g.rmax[0] - x < g.maxlink ||
            y - g.rmin[1] < g.maxlink || g.rmax[1] - y < g.maxlink ||
            z - g.rmin[2] < g.maxlink || g.rmax[2] - z < g.maxlink)
          atomicOr(warn + ci, 1u);
      }
    }
    const bool h = warp_segments<NS>(ci, v);
    if (h && ci != kNone) {
      double *s = sums + (uint64_t)ci * NS;
#pragma unroll
      for (int c = 0; c < NS; c++) atomicAdd(s + c, v[c]);
    }
  }
}

// Ownership (Checkhalo, FOF.c:394-401): centre of mass by division, kept iff
// inside [lo, hi) on every axis.
template <int NS>
__global__ void __launch_bounds__(kT) k_owned(const double *__restrict__ sums,
                                              const uint32_t *__restrict__ cand_root,
                                              const uint32_t *__restrict__ count,
                                              const uint32_t *__restrict__ ncand, Geom g,
                                              uint32_t *__restrict__ own) {
  const uint32_t nc = *ncand;
  for (int64_t c = gtid(); c < nc; c += gstride()) {
    const double n = (double)count[cand_root[c]];
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double com = __ddiv_rn(sums[(uint64_t)c * NS + a], n);
      ok &= (com >= g.lo[a]) && (com < g.hi[a]);
    }
    own[c] = ok ? 1u : 0u;
  }
}

__global__ void __launch_bounds__(kT) k_own_list(const uint32_t *__restrict__ own,
                                                 const uint32_t *__restrict__ own_scan,
                                                 const uint32_t *__restrict__ cand_root,
                                                 const uint32_t *__restrict__ head,
                                                 const uint32_t *__restrict__ ncand,
                                                 uint32_t *__restrict__ okeys,
                                                 uint32_t *__restrict__ ovals) {
  const uint32_t nc = *ncand;
  for (int64_t c = gtid(); c < nc; c += gstride()) {
    if (!own[c]) continue;
    okeys[own_scan[c]] = head[cand_root[c]];
    ovals[own_scan[c]] = (uint32_t)c;
  }
}

// Halo records (Output_Halos, FOF.c:836-872): means by the reciprocal of n,
// second-moment combinations as written there, all in double, then float.
template <int NS>
__global__ void __launch_bounds__(kT) k_catalog(const uint32_t *__restrict__ okeys,
                                                const uint32_t *__restrict__ ovals,
                                                const uint32_t *__restrict__ nown,
                                                const double *__restrict__ sums,
                                                const uint32_t *__restrict__ cand_root,
                                                const uint32_t *__restrict__ count,
                                                const uint32_t *__restrict__ warn, Geom g,
                                                float *__restrict__ props,
                                                uint32_t *__restrict__ head_out,
                                                uint32_t *__restrict__ cat_of_cand,
                                                unsigned long long *n_warn) {
  const uint32_t nh = *nown;
  for (int64_t h = gtid(); h < nh; h += gstride()) {
    const uint32_t c = ovals[h];
    const uint32_t n = count[cand_root[c]];
    const double *s = sums + (uint64_t)c * NS;
    const double inv = __ddiv_rn(1.0, (double)n);
    float *rec = props + (uint64_t)h * g.hs;
    int o = 0;
    rec[o++] = (float)n;
    for (int q = 0; q < 6; q++) rec[o++] = __double2float_rn(__dmul_rn(s[q], inv));
    int m = 6;
    if (g.props & 1) {
      const double xx = s[m], yy = s[m + 1], zz = s[m + 2], xy = s[m + 3], xz = s[m + 4],
                   yz = s[m + 5];
      const double X = s[0], Y = s[1], Z = s[2];
      rec[o++] = __double2float_rn(__dsub_rn(__dadd_rn(yy, zz), __dmul_rn(inv, __dadd_rn(__dmul_rn(Y, Y), __dmul_rn(Z, Z)))));
      rec[o++] = __double2float_rn(__dsub_rn(__dadd_rn(xx, zz), __dmul_rn(inv, __dadd_rn(__dmul_rn(X, X), __dmul_rn(Z, Z)))));
      rec[o++] = __double2float_rn(__dsub_rn(__dadd_rn(xx, yy), __dmul_rn(inv, __dadd_rn(__dmul_rn(X, X), __dmul_rn(Y, Y)))));
      rec[o++] = __double2float_rn(__dsub_rn(__dmul_rn(__dmul_rn(inv, X), Y), xy));
      rec[o++] = __double2float_rn(__dsub_rn(__dmul_rn(__dmul_rn(inv, X), Z), xz));
      rec[o++] = __double2float_rn(__dsub_rn(__dmul_rn(__dmul_rn(inv, Y), Z), yz));
      m += 6;
    }
    if (g.props & 2) {
      const double VX = s[3], VY = s[4], VZ = s[5];
      const double A[6] = {s[m], s[m + 1], s[m + 2], s[m + 3], s[m + 4], s[m + 5]};
      const double P[6] = {__dmul_rn(VX, VX), __dmul_rn(VY, VY), __dmul_rn(VZ, VZ),
                           __dmul_rn(VX, VY), __dmul_rn(VX, VZ), __dmul_rn(VY, VZ)};
      for (int q = 0; q < 6; q++)
        rec[o++] = __double2float_rn(__dmul_rn(__dsub_rn(A[q], __dmul_rn(P[q], inv)), inv));
    }
    head_out[h] = okeys[h];
    cat_of_cand[c] = (uint32_t)h;
    if (warn[c]) atomicAdd(n_warn, 1ull);
  }
}

// Membership per input particle: the owned halo holding it (or one of its
// images) -- the lowest catalog index when a halo wider than the ghost shell
// leaves two owned copies -- then, in a second pass, the processing index
// of that copy and its stored coordinates.
template <class PT>
__global__ void __launch_bounds__(kT) k_member(const uint32_t *__restrict__ run_of,
                                               const uint32_t *__restrict__ parent,
                                               const uint32_t *__restrict__ cand_of_root,
                                               const uint32_t *__restrict__ cat_of_cand,
                                               const SPos<PT> *__restrict__ spos, int64_t np,
                                               unsigned long long *__restrict__ member) {
  for (int64_t i = gtid(); i < np; i += gstride()) {
    const uint32_t ci = cand_of_root[parent[run_of[i]]];
    if (ci == kNone) continue;
    const uint32_t h = cat_of_cand[ci];
    if (h == kNone) continue;
    atomicMin(member + spos[i].src, (unsigned long long)h);
  }
}

template <class PT>
__global__ void __launch_bounds__(kT) k_member_copy(
    const uint32_t *__restrict__ run_of, const uint32_t *__restrict__ parent,
    const uint32_t *__restrict__ cand_of_root, const uint32_t *__restrict__ cat_of_cand,
    const SPos<PT> *__restrict__ spos, const uint32_t *__restrict__ perm, int64_t np,
    const unsigned long long *__restrict__ member, uint32_t *__restrict__ member_proc,
    float *__restrict__ member_pos, Counters *ctr) {
  for (int64_t i = gtid(); i < np; i += gstride()) {
    const uint32_t ci = cand_of_root[parent[run_of[i]]];
    if (ci == kNone) continue;
    const uint32_t h = cat_of_cand[ci];
    if (h == kNone) continue;
    const SPos<PT> p = spos[i];
    if (member[p.src] == (unsigned long long)h) {
      member_proc[p.src] = perm[i];
      member_pos[3 * (uint64_t)p.src] = (float)p.x;
      member_pos[3 * (uint64_t)p.src + 1] = (float)p.y;
      member_pos[3 * (uint64_t)p.src + 2] = (float)p.z;
    } else {
      atomicAdd(&ctr->member_conflicts, 1ull);
    }
  }
}

int bits_for(uint64_t v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) b++;
  return b;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side of one run.
// ---------------------------------------------------------------------------

void Plan::setup_geometry(int64_t n_in) {
  const cmh_fof_params &p = params;
  Geom &g = geom;
  g = Geom{};
  double minlink = p.linklength, maxlink = p.linklength;
  if (p.varlink) {
    minlink = maxlink = ltab_host.empty() ? p.linklength : ltab_host[0];
    for (double v : ltab_host) {
      minlink = std::min(minlink, v);
      maxlink = std::max(maxlink, v);
    }
  }
  if (!(minlink > 0) || !std::isfinite(maxlink))
    fail(CMH_ERR_INVALID_ARGUMENT, "linking length must be positive and finite");
  for (int a = 0; a < 3; a++) {
    g.lo[a] = p.lo[a];
    g.hi[a] = p.hi[a];
    g.rmin[a] = p.lo[a] - p.boundary;  // startup.c:40-47
    g.rmax[a] = p.hi[a] + p.boundary;
    g.L[a] = p.hi[a] - p.lo[a];
    if (!(g.L[a] > 0)) fail(CMH_ERR_INVALID_ARGUMENT, "box extent must be positive");
  }
  g.boundary = p.boundary;
  g.linksq = p.linklength * p.linklength;  // FOF.c:60
  g.maxlink = maxlink;
  g.prune_sq = (maxlink * (1.0 + 1e-5)) * (maxlink * (1.0 + 1e-5));
  g.nphalomin = p.nphalomin;
  g.periodic = p.periodic ? 1 : 0;
  g.props = (int)(p.properties & 3u);
  g.hs = 7 + ((g.props & 1) ? 6 : 0) + ((g.props & 2) ? 6 : 0);
  band_thresholds(g.linksq, pos_dtype == CMH_FLOAT64 ? 8 : 4, &g.t_lo, &g.t_hi);
  // fine cell: any two points of a cell are closer than minlink
  g.h = minlink * (1.0 - 0x1p-20) / std::sqrt(3.0);
  g.inv_h = 1.0 / g.h;
  g.W = (int)std::floor(maxlink / g.h * (1.0 + 1e-6)) + 1;
  double vol = 1.0;
  for (int a = 0; a < 3; a++) {
    g.G[a] = (int)std::floor((g.rmax[a] - g.rmin[a]) / g.h) + 2;
    if (g.G[a] >= (1 << 21)) fail(CMH_ERR_CAPACITY, "more than 2^21 fine cells along an axis");
    vol *= (g.rmax[a] - g.rmin[a]);
  }
  int k = p.cell_factor;
  if (k <= 0) {
    // one top cell per particle on average, as the reference's lcell = L/Px
    const double sep = std::cbrt(vol / std::max<double>((double)n_in, 1.0));
    k = (int)std::lround(sep / g.h);
  }
  k = std::max(k, g.W);
  while (true) {
    uint64_t T = 1;
    for (int a = 0; a < 3; a++) {
      g.T[a] = (g.G[a] + k - 1) / k;
      T *= (uint64_t)g.T[a];
    }
    const uint64_t k3 = (uint64_t)k * k * k;
    if (T < (1ull << 31) && (T * k3) < (1ull << 62)) {
      g.k = k;
      g.k3 = k3;
      n_top = T;
      key_bits = bits_for(T * k3 - 1);
      break;
    }
    k++;
  }
}

template <class PT, class VT>
void Plan::run_typed(const cmh_particles &parts, bool want_member, cudaStream_t s) {
  const int64_t n = parts.n;
  const PT *pos = static_cast<const PT *>(parts.pos);
  const VT *vel = static_cast<const VT *>(parts.vel);
  Geom &g = geom;
  stats = cmh_stats{};
  stats.n_in = n;
  const long long launches0 = g_launches;
  CMH_CUDA(cudaEventRecord(ev0, s));

  // scalars: [0] n_kept [1] n_images [2] R [3] n_dense [4] n_cand [5] n_own
  scal.ensure(16 * sizeof(uint32_t));
  ctr.ensure(sizeof(Counters) + 2 * sizeof(unsigned long long));
  uint32_t *sc = scal.as<uint32_t>();
  Counters *c = ctr.as<Counters>();
  unsigned long long *extra = reinterpret_cast<unsigned long long *>(c + 1);  // ngroups, nwarn
  CMH_CUDA(cudaMemsetAsync(scal.p, 0, 16 * sizeof(uint32_t), s));
  CMH_CUDA(cudaMemsetAsync(ctr.p, 0, sizeof(Counters) + 2 * sizeof(unsigned long long), s));
  if (g.varlink) fail(CMH_ERR_INVALID_ARGUMENT, "variable linking length is not built yet");

  // ---- ingest ----
  const int64_t nn = std::max<int64_t>(n, 1);
  b_keep.ensure(nn * 4);
  b_nimg.ensure(nn * 4);
  b_keep_scan.ensure(nn * 4);
  b_img_scan.ensure(nn * 4);
  if (n > 0) {
    k_ingest_count<PT><<<grid_for(n, kT), kT, 0, s>>>(pos, n, g, b_keep.as<uint32_t>(),
                                                      b_nimg.as<uint32_t>());
    CMH_LAUNCHED();
  }
  exclusive_scan_u32(b_keep.as<uint32_t>(), b_keep_scan.as<uint32_t>(), n, sc + 0, scan_tmp, s);
  exclusive_scan_u32(b_nimg.as<uint32_t>(), b_img_scan.as<uint32_t>(), n, sc + 1, scan_tmp, s);
  CMH_CUDA(cudaMemcpyAsync(h_scal, sc, 16 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CMH_CUDA(cudaStreamSynchronize(s));
  const int64_t n_kept = h_scal[0], n_img = h_scal[1];
  const int64_t np = n_kept + n_img;
  stats.n_out = n - n_kept;
  stats.n_images = n_img;
  stats.n_proc = np;
  if (np >= (int64_t)0xffffffffll) fail(CMH_ERR_CAPACITY, "more than 2^32-2 processed particles");

  // ---- keys, sort, runs ----
  const int64_t npp = std::max<int64_t>(np, 1);
  b_keys.ensure(npp * 8);
  b_keys_alt.ensure(npp * 8);
  b_vals.ensure(npp * 4);
  b_vals_alt.ensure(npp * 4);
  b_ppos.ensure(npp * sizeof(SPos<PT>));
  b_spos.ensure(npp * sizeof(SPos<PT>));
  b_run_of.ensure(npp * 4);
  if (n > 0) {
    k_ingest_emit<PT><<<grid_for(n, kT), kT, 0, s>>>(
        pos, n, g, b_keep.as<uint32_t>(), b_keep_scan.as<uint32_t>(), b_img_scan.as<uint32_t>(),
        b_nimg.as<uint32_t>(), sc + 0, b_keys.as<uint64_t>(), b_vals.as<uint32_t>(), b_ppos.as<SPos<PT>>());
    CMH_LAUNCHED();
  }
  CMH_CUDA(cudaEventRecord(stage_ev[0], s));
  radix_sort_u64_u32(b_keys.as<uint64_t>(), b_vals.as<uint32_t>(), b_keys_alt.as<uint64_t>(),
                     b_vals_alt.as<uint32_t>(), np, key_bits, sort_tmp, scan_tmp, s);
  CMH_CUDA(cudaEventRecord(stage_ev[1], s));
  uint32_t *flag = b_keys_alt.as<uint32_t>();  // reuse: [flag | run_scan]
  uint32_t *run_scan = flag + npp;
  if (np > 0) {
    k_gather_flags<PT><<<grid_for(np, kT), kT, 0, s>>>(b_keys.as<uint64_t>(), b_vals.as<uint32_t>(),
                                                       b_ppos.as<SPos<PT>>(), b_spos.as<SPos<PT>>(),
                                                       flag, np);
    CMH_LAUNCHED();
  }
  exclusive_scan_u32(flag, run_scan, np, sc + 2, scan_tmp, s);
  CMH_CUDA(cudaMemcpyAsync(h_scal + 2, sc + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CMH_CUDA(cudaStreamSynchronize(s));
  const int64_t R = h_scal[2];
  stats.n_cells = R;
  const int64_t RR = std::max<int64_t>(R, 1);
  b_run_start.ensure((RR + 1) * 4);
  b_run_g.ensure(RR * 8);
  if (np > 0) {
    k_runs<<<grid_for(np, kT), kT, 0, s>>>(b_keys.as<uint64_t>(), flag, run_scan, np, g,
                                           b_run_of.as<uint32_t>(), b_run_start.as<uint32_t>(),
                                           b_run_g.as<uint64_t>(), sc + 2);
    CMH_LAUNCHED();
  }
  // ---- top-cell ranges and dense maps ----
  b_top_first.ensure(n_top * 4);
  b_top_end.ensure(n_top * 4);
  b_top_slot.ensure(n_top * 4);
  CMH_CUDA(cudaMemsetAsync(b_top_first.p, 0, n_top * 4, s));
  CMH_CUDA(cudaMemsetAsync(b_top_end.p, 0, n_top * 4, s));
  const unsigned gr = grid_for(RR, kT);
  k_top_ranges<<<gr, kT, 0, s>>>(b_run_g.as<uint64_t>(), g, sc + 2, b_top_first.as<uint32_t>(),
                                 b_top_end.as<uint32_t>());
  CMH_LAUNCHED();
  b_rtmp1.ensure(RR * 4);
  b_rtmp2.ensure(RR * 4);
  k_dense_flags<<<gr, kT, 0, s>>>(b_run_g.as<uint64_t>(), g, sc + 2, b_top_first.as<uint32_t>(),
                                  b_top_end.as<uint32_t>(), dense_min, b_rtmp1.as<uint32_t>());
  CMH_LAUNCHED();
  exclusive_scan_u32(b_rtmp1.as<uint32_t>(), b_rtmp2.as<uint32_t>(), R, sc + 3, scan_tmp, s);
  CMH_CUDA(cudaMemcpyAsync(h_scal + 3, sc + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CMH_CUDA(cudaStreamSynchronize(s));
  const int64_t nd = h_scal[3];
  b_maps.ensure(std::max<int64_t>(nd, 1) * g.k3 * 4);
  b_dense_range.ensure(std::max<int64_t>(nd, 1) * sizeof(uint2));
  if (nd > 0) {
    CMH_CUDA(cudaMemsetAsync(b_maps.p, 0xff, nd * g.k3 * 4, s));
    k_dense_maps<<<gr, kT, 0, s>>>(b_run_g.as<uint64_t>(), g, sc + 2, b_top_first.as<uint32_t>(),
                                   b_top_end.as<uint32_t>(), b_rtmp1.as<uint32_t>(),
                                   b_rtmp2.as<uint32_t>(), dense_min, b_top_slot.as<uint32_t>(),
                                   b_dense_range.as<uint2>(), b_maps.as<int32_t>());
    CMH_LAUNCHED();
  }
  // ---- befriending ----
  b_parent.ensure(RR * 4);
  k_iota<<<gr, kT, 0, s>>>(b_parent.as<uint32_t>(), sc + 2);
  CMH_LAUNCHED();
  CMH_CUDA(cudaEventRecord(stage_ev[2], s));
  // dense top cells joined inside (CTA each), then a fast path for every
  // cell, a queue of the crowded ones and a warp path for those
  uint32_t *queue = b_rtmp1.as<uint32_t>();  // free again after the dense maps
  // sc[6] queue length, sc[7..9] work counters of the dense and warp passes
  CMH_CUDA(cudaMemsetAsync(sc + 6, 0, 4 * sizeof(uint32_t), s));
  const unsigned gw = grid_for(RR * 32, kT);  // one warp per queued cell
  const size_t dsm = (size_t)g.k3 * sizeof(uint32_t);
  const unsigned gd = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nd, (int64_t)kSMs * 16));
#define CMH_BEFRIEND(FP)                                                                      \
  if (nd > 0) {                                                                               \
    CMH_CUDA(cudaFuncSetAttribute(k_befriend_dense<PT, FP>,                                   \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));    \
    k_befriend_dense<PT, FP><<<gd, 128, dsm, s>>>(g, b_run_start.as<uint32_t>(),              \
                                                  b_run_g.as<uint64_t>(),                     \
                                                  b_dense_range.as<uint2>(), sc + 3, sc + 7,  \
                                                  b_maps.as<int32_t>(), b_spos.as<SPos<PT>>(), \
                                                  b_parent.as<uint32_t>(), c);                \
    CMH_LAUNCHED();                                                                           \
  }                                                                                           \
  k_befriend_simple<PT, FP><<<gr, kT, 0, s>>>(g, b_run_start.as<uint32_t>(),                 \
                                              b_run_g.as<uint64_t>(), sc + 2,                 \
                                              b_top_first.as<uint32_t>(),                     \
                                              b_top_end.as<uint32_t>(), dense_min,            \
                                              b_spos.as<SPos<PT>>(), b_parent.as<uint32_t>(), \
                                              queue, sc + 6, c);                              \
  CMH_LAUNCHED();                                                                             \
  k_befriend<PT, FP, 0><<<gw, kT, 0, s>>>(                                                    \
      g, b_run_start.as<uint32_t>(), b_run_g.as<uint64_t>(), queue, sc + 6, sc + 8,          \
      b_top_first.as<uint32_t>(), b_top_end.as<uint32_t>(), b_top_slot.as<uint32_t>(),       \
      b_maps.as<int32_t>(), dense_min, b_spos.as<SPos<PT>>(), b_parent.as<uint32_t>(), c);  \
  CMH_LAUNCHED();                                                                             \
  k_compress<<<gr, kT, 0, s>>>(b_parent.as<uint32_t>(), sc + 2);                              \
  CMH_LAUNCHED();                                                                             \
  k_befriend<PT, FP, 1><<<gw, kT, 0, s>>>(                                                    \
      g, b_run_start.as<uint32_t>(), b_run_g.as<uint64_t>(), queue, sc + 6, sc + 9,          \
      b_top_first.as<uint32_t>(), b_top_end.as<uint32_t>(), b_top_slot.as<uint32_t>(),       \
      b_maps.as<int32_t>(), dense_min, b_spos.as<SPos<PT>>(), b_parent.as<uint32_t>(), c);  \
  CMH_LAUNCHED()
  if (fp32) {
    CMH_BEFRIEND(true);
  } else {
    CMH_BEFRIEND(false);
  }
#undef CMH_BEFRIEND
  k_compress<<<gr, kT, 0, s>>>(b_parent.as<uint32_t>(), sc + 2);
  CMH_LAUNCHED();
  CMH_CUDA(cudaEventRecord(stage_ev[3], s));

  // ---- groups, candidates ----
  b_count.ensure(RR * 4);
  b_head.ensure(RR * 4);
  b_cand_of_root.ensure(RR * 4);
  CMH_CUDA(cudaMemsetAsync(b_count.p, 0, RR * 4, s));
  CMH_CUDA(cudaMemsetAsync(b_head.p, 0xff, RR * 4, s));
  CMH_CUDA(cudaMemsetAsync(b_cand_of_root.p, 0xff, RR * 4, s));
  if (np > 0) {
    k_group_count<<<grid_for(np, kT), kT, 0, s>>>(b_run_of.as<uint32_t>(), b_parent.as<uint32_t>(),
                                                  b_vals.as<uint32_t>(), np, b_count.as<uint32_t>(),
                                                  b_head.as<uint32_t>());
    CMH_LAUNCHED();
  }
  k_cand_flags<<<gr, kT, 0, s>>>(b_parent.as<uint32_t>(), b_count.as<uint32_t>(), sc + 2,
                                 g.nphalomin, b_rtmp1.as<uint32_t>(), extra + 0);
  CMH_LAUNCHED();
  exclusive_scan_u32(b_rtmp1.as<uint32_t>(), b_rtmp2.as<uint32_t>(), R, sc + 4, scan_tmp, s);
  CMH_CUDA(cudaMemcpyAsync(h_scal + 4, sc + 4, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CMH_CUDA(cudaStreamSynchronize(s));
  const int64_t nc = h_scal[4];
  const int64_t ncc = std::max<int64_t>(nc, 1);
  b_cand_root.ensure(ncc * 4);
  k_cand_list<<<gr, kT, 0, s>>>(b_rtmp1.as<uint32_t>(), b_rtmp2.as<uint32_t>(), sc + 2,
                                b_cand_of_root.as<uint32_t>(), b_cand_root.as<uint32_t>());
  CMH_LAUNCHED();
  CMH_CUDA(cudaEventRecord(stage_ev[4], s));

  // ---- property sums, ownership, catalog ----
  const int NS = 6 + ((g.props & 1) ? 6 : 0) + ((g.props & 2) ? 6 : 0);
  b_sums.ensure(ncc * NS * 8);
  b_warn.ensure(ncc * 4);
  CMH_CUDA(cudaMemsetAsync(b_sums.p, 0, ncc * NS * 8, s));
  CMH_CUDA(cudaMemsetAsync(b_warn.p, 0, ncc * 4, s));
  if (np > 0 && nc > 0) {
    const unsigned gp = grid_for(np, kT);
    if (NS == 6)
      k_group_sums<PT, VT, 6><<<gp, kT, 0, s>>>(b_run_of.as<uint32_t>(), b_parent.as<uint32_t>(),
                                                b_cand_of_root.as<uint32_t>(), b_spos.as<SPos<PT>>(),
                                                vel, np, g, b_sums.as<double>(), b_warn.as<uint32_t>());
    else if (NS == 12)
      k_group_sums<PT, VT, 12><<<gp, kT, 0, s>>>(b_run_of.as<uint32_t>(), b_parent.as<uint32_t>(),
                                                 b_cand_of_root.as<uint32_t>(), b_spos.as<SPos<PT>>(),
                                                 vel, np, g, b_sums.as<double>(), b_warn.as<uint32_t>());
    else
      k_group_sums<PT, VT, 18><<<gp, kT, 0, s>>>(b_run_of.as<uint32_t>(), b_parent.as<uint32_t>(),
                                                 b_cand_of_root.as<uint32_t>(), b_spos.as<SPos<PT>>(),
                                                 vel, np, g, b_sums.as<double>(), b_warn.as<uint32_t>());
    CMH_LAUNCHED();
  }
  CMH_CUDA(cudaEventRecord(stage_ev[5], s));
  b_own.ensure(ncc * 4);
  b_own_scan.ensure(ncc * 4);
  const unsigned gc = grid_for(ncc, kT);
  if (NS == 6)
    k_owned<6><<<gc, kT, 0, s>>>(b_sums.as<double>(), b_cand_root.as<uint32_t>(),
                                 b_count.as<uint32_t>(), sc + 4, g, b_own.as<uint32_t>());
  else if (NS == 12)
    k_owned<12><<<gc, kT, 0, s>>>(b_sums.as<double>(), b_cand_root.as<uint32_t>(),
                                  b_count.as<uint32_t>(), sc + 4, g, b_own.as<uint32_t>());
  else
    k_owned<18><<<gc, kT, 0, s>>>(b_sums.as<double>(), b_cand_root.as<uint32_t>(),
                                  b_count.as<uint32_t>(), sc + 4, g, b_own.as<uint32_t>());
  CMH_LAUNCHED();
  exclusive_scan_u32(b_own.as<uint32_t>(), b_own_scan.as<uint32_t>(), nc, sc + 5, scan_tmp, s);
  CMH_CUDA(cudaMemcpyAsync(h_scal + 5, sc + 5, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CMH_CUDA(cudaStreamSynchronize(s));
  const int64_t nh = h_scal[5];
  const int64_t nhh = std::max<int64_t>(nh, 1);
  b_okeys.ensure(nhh * 4);
  b_ovals.ensure(nhh * 4);
  b_okeys_alt.ensure(nhh * 4);
  b_ovals_alt.ensure(nhh * 4);
  k_own_list<<<gc, kT, 0, s>>>(b_own.as<uint32_t>(), b_own_scan.as<uint32_t>(),
                               b_cand_root.as<uint32_t>(), b_head.as<uint32_t>(), sc + 4,
                               b_okeys.as<uint32_t>(), b_ovals.as<uint32_t>());
  CMH_LAUNCHED();
  radix_sort_u32_u32(b_okeys.as<uint32_t>(), b_ovals.as<uint32_t>(), b_okeys_alt.as<uint32_t>(),
                     b_ovals_alt.as<uint32_t>(), nh, bits_for((uint64_t)npp), sort_tmp, scan_tmp, s);
  b_props.ensure(nhh * g.hs * 4);
  b_head_out.ensure(nhh * 4);
  b_cat_of_cand.ensure(ncc * 4);
  CMH_CUDA(cudaMemsetAsync(b_cat_of_cand.p, 0xff, ncc * 4, s));
  const unsigned gh = grid_for(nhh, kT);
#define CMH_CATALOG(NSV)                                                                    \
  k_catalog<NSV><<<gh, kT, 0, s>>>(b_okeys.as<uint32_t>(), b_ovals.as<uint32_t>(), sc + 5, \
                                   b_sums.as<double>(), b_cand_root.as<uint32_t>(),         \
                                   b_count.as<uint32_t>(), b_warn.as<uint32_t>(), g,        \
                                   b_props.as<float>(), b_head_out.as<uint32_t>(),          \
                                   b_cat_of_cand.as<uint32_t>(), extra + 1)
  if (NS == 6) CMH_CATALOG(6);
  else if (NS == 12) CMH_CATALOG(12);
  else CMH_CATALOG(18);
#undef CMH_CATALOG
  CMH_LAUNCHED();
  CMH_CUDA(cudaEventRecord(stage_ev[6], s));
  if (want_member) {
    b_member.ensure(nn * 8);
    b_member_proc.ensure(nn * 4);
    b_member_pos.ensure(nn * 12);
    CMH_CUDA(cudaMemsetAsync(b_member.p, 0xff, nn * 8, s));
    CMH_CUDA(cudaMemsetAsync(b_member_proc.p, 0xff, nn * 4, s));
    CMH_CUDA(cudaMemsetAsync(b_member_pos.p, 0, nn * 12, s));
    if (np > 0) {
      k_member<PT><<<grid_for(np, kT), kT, 0, s>>>(
          b_run_of.as<uint32_t>(), b_parent.as<uint32_t>(), b_cand_of_root.as<uint32_t>(),
          b_cat_of_cand.as<uint32_t>(), b_spos.as<SPos<PT>>(), np,
          b_member.as<unsigned long long>());
      CMH_LAUNCHED();
      k_member_copy<PT><<<grid_for(np, kT), kT, 0, s>>>(
          b_run_of.as<uint32_t>(), b_parent.as<uint32_t>(), b_cand_of_root.as<uint32_t>(),
          b_cat_of_cand.as<uint32_t>(), b_spos.as<SPos<PT>>(), b_vals.as<uint32_t>(), np,
          b_member.as<unsigned long long>(), b_member_proc.as<uint32_t>(),
          b_member_pos.as<float>(), c);
      CMH_LAUNCHED();
    }
  }
  CMH_CUDA(cudaEventRecord(ev1, s));
  // ---- statistics ----
  struct {
    Counters c;
    unsigned long long ngroups, nwarn;
  } hc;
  CMH_CUDA(cudaMemcpyAsync(&hc, ctr.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
  CMH_CUDA(cudaStreamSynchronize(s));
  if (hc.c.uf_giveups)
    fail(CMH_ERR_DEVICE_TIMEOUT, "union-find retry loop reached its iteration cap");
  float ms = 0;
  CMH_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  {
    cudaEvent_t b[9] = {ev0, stage_ev[0], stage_ev[1], stage_ev[2], stage_ev[3],
                        stage_ev[4], stage_ev[5], stage_ev[6], ev1};
    for (int q = 0; q < 8; q++) CMH_CUDA(cudaEventElapsedTime(&stats.stage_ms[q], b[q], b[q + 1]));
  }
  stats.n_launches = (int32_t)(g_launches - launches0);
  stats.n_groups = (int64_t)hc.ngroups;
  stats.n_candidates = nc;
  stats.nhalos = nh;
  stats.n_edge_warn = (int64_t)hc.nwarn;
  stats.n_pair_tests = (int64_t)hc.c.pair_tests;
  stats.n_rechecks = (int64_t)hc.c.rechecks;
  stats.n_cell_pairs = (int64_t)hc.c.cand_pairs;
  stats.n_root_skips = (int64_t)hc.c.root_skips;
  stats.n_unions = (int64_t)hc.c.unions;
  stats.n_find_steps = (int64_t)hc.c.find_steps;
  stats.n_scan_iters = (int64_t)hc.c.scan_iters;
  stats.n_window_iters = (int64_t)hc.c.window_iters;
  stats.n_dense_tops = (int64_t)nd;
  stats.n_member_conflicts = (int64_t)hc.c.member_conflicts;
  stats.cell_factor = g.k;
  stats.key_bits = key_bits;
  stats.ms_total = ms;
  out_nhalos = nh;
}

void Plan::run(const cmh_particles &parts, bool want_member, cudaStream_t s) {
  CMH_CUDA(cudaSetDevice(device));
  setup_geometry(parts.n);
  const bool pd = parts.pos_dtype == CMH_FLOAT64, vd = parts.vel_dtype == CMH_FLOAT64;
  if (pd && vd) run_typed<double, double>(parts, want_member, s);
  else if (pd) run_typed<double, float>(parts, want_member, s);
  else if (vd) run_typed<float, double>(parts, want_member, s);
  else run_typed<float, float>(parts, want_member, s);
}

}  // namespace cmh
