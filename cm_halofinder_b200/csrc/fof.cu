// The FoF hot path on one B200: ingest + periodic images, cell keys, radix
// sort, fine-cell runs, befriending with a lock-free union-find, and the
// segmented reductions that produce the halo catalog.  A run holds one or
// many independent domains ("boxes"); all of them go through the same
// launches (one sort, one befriending pass, one reduction for the batch), and
// no size is read back by the host until the run is issued, so a run can be
// captured in a CUDA graph and replayed.
//
// Reference: src_v2/FOF.c (FOF, Befriend, Checkhalo, Output_Halos property
// sums) and src_v2/read_data.c:409-424,785-816 (domain filter, ghost wrap).
//
// Cells.  Particles are keyed by a fine cell of side h <= l_min / sqrt(3)
// (with a 2^-20 margin): two particles in the same fine cell are closer than
// the linking length whatever their position inside it, so every occupied
// fine cell is one connected piece and union-find runs over cells, not
// particles.  Fine cells are grouped k^3 to a top cell; the sort key is
// (top cell, fine cell inside it), each box's top cells numbered after the
// previous box's, so a top cell's fine cells are contiguous and the
// befriending step visits the 27-cell top stencil (self + 13 forward
// neighbours), exactly the cell loop of FOF.c:96-161 one level up.
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
#include <cstring>
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

// Index of the last entry of base[0..nb) that is <= x (base[0] == 0).
__device__ __forceinline__ int box_search(const uint64_t *base, int nb, uint64_t x) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Copies the boxes' first input index (or first top cell) into shared memory.
__device__ __forceinline__ void load_bases(const BoxDev *boxes, int nbox, uint64_t *s, bool tops) {
  for (int b = threadIdx.x; b < nbox; b += blockDim.x) s[b] = tops ? boxes[b].top_base : boxes[b].in_base;
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Ingest: domain filter (read_data.c:409-424) and periodic images.
// ---------------------------------------------------------------------------

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
__device__ __forceinline__ void load_pos(const BoxDev &bx, uint64_t li, double x[3]) {
  const PT *pos = static_cast<const PT *>(bx.pos);
  x[0] = as_d(pos[3 * li]);
  x[1] = as_d(pos[3 * li + 1]);
  x[2] = as_d(pos[3 * li + 2]);
}

// Keep flag (bit 0: inside the domain) and image count (bits 1..) of a
// particle at x.
// A shift by -L (+L) can only stay in the shell for x within the boundary
// size of the upper (lower) face: farther in, x -+ L lies beyond the shell by
// more than the margin, which is far above the rounding of x -+ L to PT, so
// only particles within the margin are tested exactly.
template <class PT>
__device__ __forceinline__ uint32_t ingest_flags(const Geom &g, const double x[3]) {
  if (!in_domain(g, x)) return 0u;
  uint32_t cnt = 0;
  if (g.periodic) {
    int opt[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double margin = g.boundary + 1e-5 * (fabs(g.lo[a]) + fabs(g.hi[a]) + g.boundary);
      double c;
      opt[a] = 1;
      if (g.hi[a] - x[a] <= margin) opt[a] += (int)image_coord<PT>(g, x[a], a, -1, &c);
      if (x[a] - g.lo[a] <= margin) opt[a] += (int)image_coord<PT>(g, x[a], a, 1, &c);
    }
    cnt = (uint32_t)(opt[0] * opt[1] * opt[2] - 1);
  }
  return 1u | (cnt << 1);
}

// Two particles per thread and step (i and i + stride), both positions
// loaded before either is tested, so that each step waits on memory once.
template <class PT>
__global__ void __launch_bounds__(kT) k_ingest_count(const BoxDev *__restrict__ boxes, int nbox,
                                                     int64_t n, uint32_t *__restrict__ keep,
                                                     uint32_t *__restrict__ nimg) {
  __shared__ uint64_t s_base[kMaxBoxes];
  load_bases(boxes, nbox, s_base, false);
  const int64_t st = gstride();
  for (int64_t i0 = gtid(); i0 < n; i0 += 2 * st) {
    const int64_t i1 = i0 + st;
    const bool has1 = i1 < n;
    const int b0 = box_search(s_base, nbox, (uint64_t)i0);
    const int b1 = has1 ? box_search(s_base, nbox, (uint64_t)i1) : b0;
    double x0[3], x1[3] = {0.0, 0.0, 0.0};
    load_pos<PT>(boxes[b0], (uint64_t)i0 - s_base[b0], x0);
    if (has1) load_pos<PT>(boxes[b1], (uint64_t)i1 - s_base[b1], x1);
    const uint32_t f0 = ingest_flags<PT>(boxes[b0].g, x0);
    keep[i0] = f0 & 1u;
    nimg[i0] = f0 >> 1;
    if (has1) {
      const uint32_t f1 = ingest_flags<PT>(boxes[b1].g, x1);
      keep[i1] = f1 & 1u;
      nimg[i1] = f1 >> 1;
    }
  }
}

// Per box: kept and image counts, and the first processing index of the box
// (its kept particles, then its images).  Sets the run's processed count,
// clamped to the capacity `np_cap`.
__global__ void k_box_totals(const BoxDev *__restrict__ boxes, int nbox, int64_t n,
                             const uint32_t *__restrict__ keep_scan,
                             const uint32_t *__restrict__ img_scan, DevScal *sc,
                             uint32_t *__restrict__ boxd, uint32_t np_cap) {
  // boxd layout: [kept_before | img_before | nkept | nimg | proc_base | halo_count | halo_base]
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint64_t acc = 0;
  for (int b = 0; b < nbox; b++) {
    const uint64_t i0 = boxes[b].in_base, i1 = i0 + boxes[b].n;
    const uint32_t k0 = i0 < (uint64_t)n ? keep_scan[i0] : sc->kept_total;
    const uint32_t k1 = i1 < (uint64_t)n ? keep_scan[i1] : sc->kept_total;
    const uint32_t m0 = i0 < (uint64_t)n ? img_scan[i0] : sc->img_total;
    const uint32_t m1 = i1 < (uint64_t)n ? img_scan[i1] : sc->img_total;
    boxd[0 * nbox + b] = k0;
    boxd[1 * nbox + b] = m0;
    boxd[2 * nbox + b] = k1 - k0;
    boxd[3 * nbox + b] = m1 - m0;
    boxd[4 * nbox + b] = (uint32_t)acc;
    acc += (uint64_t)(k1 - k0) + (m1 - m0);
  }
  const uint64_t np = acc;
  sc->np_raw = np > 0xffffffffull ? 0xffffffffu : (uint32_t)np;
  sc->np = np > np_cap ? np_cap : (uint32_t)np;
  if (np > np_cap) atomicOr(&sc->overflow, 1u);
}

// Fine-cell key of a processed particle at c: (top cell, counted over the
// run's boxes) * k^3 + the fine cell within it.  c holds the stored (PT)
// coordinates, so the fine cell can be recomputed from the stored position.
__device__ __forceinline__ uint64_t cell_key(const Geom &g, uint64_t top_base, uint64_t k3all,
                                             const double c[3]) {
  int gi[3];
#pragma unroll
  for (int a = 0; a < 3; a++) gi[a] = fine_index(c[a], g.rmin[a], g.inv_h, g.G[a]);
  const int k = g.k;
  const int t[3] = {div_k(gi[0], g), div_k(gi[1], g), div_k(gi[2], g)};
  const uint64_t top = top_base + ((uint64_t)t[2] * g.T[1] + t[1]) * g.T[0] + t[0];
  const uint64_t sub = ((uint64_t)(gi[2] - t[2] * k) * k + (gi[1] - t[1] * k)) * k + (gi[0] - t[0] * k);
  return top * k3all + sub;
}

template <class PT>
__device__ __forceinline__ void emit_one(const Geom &g, uint64_t top_base, uint64_t k3all,
                                         uint32_t p, const double c[3], uint32_t src,
                                         uint64_t *keys, uint32_t *vals, SPos<PT> *ppos) {
  keys[p] = cell_key(g, top_base, k3all, c);
  vals[p] = p;
  SPos<PT> s;
  s.x = (PT)c[0];
  s.y = (PT)c[1];
  s.z = (PT)c[2];
  s.src = src;
  ppos[p] = s;
}

// Processing order of a box: kept originals in input order, then the images
// grouped by source particle and shift code (sz+1)*9 + (sy+1)*3 + (sx+1)
// ascending.  Writes beyond the capacity are dropped (the run is then
// repeated with more room).  A warp walks 32 consecutive particles; their
// images are then emitted one per lane (32 at a time), so that image work
// is proportional to the images, not to the 26 shifts of each particle
// that has some.
template <class PT>
__global__ void __launch_bounds__(kT) k_ingest_emit(
    const BoxDev *__restrict__ boxes, int nbox, int64_t n, uint64_t k3all,
    const uint32_t *__restrict__ keep, const uint32_t *__restrict__ keep_scan,
    const uint32_t *__restrict__ img_scan, const uint32_t *__restrict__ nimg,
    const uint32_t *__restrict__ boxd, uint32_t np_cap, uint64_t *__restrict__ keys,
    uint32_t *__restrict__ vals, SPos<PT> *__restrict__ ppos) {
  __shared__ uint64_t s_base[kMaxBoxes];
  load_bases(boxes, nbox, s_base, false);
  const int lane = threadIdx.x & 31;
  for (int64_t w0 = gtid() - lane; w0 < n; w0 += gstride()) {
    const int64_t i = w0 + lane;
    int b = 0;
    double x[3] = {0.0, 0.0, 0.0};
    uint32_t q0 = 0, ic = 0, opts = 0;
    if (i < n) {
      // every load of the particle is issued before any is used
      b = box_search(s_base, nbox, (uint64_t)i);
      const BoxDev &bx = boxes[b];
      const uint32_t kp = keep[i], ks = keep_scan[i], is = img_scan[i], ni = nimg[i];
      load_pos<PT>(bx, (uint64_t)i - s_base[b], x);
      if (kp) {
        const uint32_t pbase = boxd[4 * nbox + b];
        const uint32_t p = pbase + (ks - boxd[0 * nbox + b]);
        if (p < np_cap) emit_one<PT>(bx.g, bx.top_base, k3all, p, x, (uint32_t)i, keys, vals, ppos);
        if (bx.g.periodic && ni != 0) {
          ic = ni;
          q0 = pbase + boxd[2 * nbox + b] + (is - boxd[1 * nbox + b]);
          // per axis: whether the -1 / +1 shift stays in the shell
#pragma unroll
          for (int a = 0; a < 3; a++) {
            double c;
            opts |= (uint32_t)image_coord<PT>(bx.g, x[a], a, -1, &c) << (2 * a);
            opts |= (uint32_t)image_coord<PT>(bx.g, x[a], a, 1, &c) << (2 * a + 1);
          }
        }
      }
    }
    // The warp's images, one per lane, in (particle, shift code) order: a
    // particle's images are the product of its per-axis options (-1 | 0 | +1
    // where the shifted coordinate stays in the shell) without (0, 0, 0),
    // in ascending code (sz+1)*9 + (sy+1)*3 + (sx+1), so the r-th one is
    // the r-th (r+1-th past (0, 0, 0)) entry of that product in z, y, x order.
    uint32_t inc = ic;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += o;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
    for (uint32_t m0 = 0; m0 < total; m0 += 32) {
      const uint32_t m = m0 + (uint32_t)lane;
      // source lane: the number of lanes whose inclusive count is <= m
      int own = 0;
#pragma unroll
      for (int st = 16; st >= 1; st >>= 1)
        if (__shfl_sync(0xffffffffu, inc, own + st - 1) <= m) own += st;
      const uint32_t o_inc = __shfl_sync(0xffffffffu, inc, own);
      const uint32_t o_ic = __shfl_sync(0xffffffffu, ic, own);
      const uint32_t o_opts = __shfl_sync(0xffffffffu, opts, own);
      const uint32_t o_q0 = __shfl_sync(0xffffffffu, q0, own);
      const int o_b = __shfl_sync(0xffffffffu, b, own);
      const int64_t o_i = __shfl_sync(0xffffffffu, i, own);
      double ox[3];
#pragma unroll
      for (int a = 0; a < 3; a++) ox[a] = __shfl_sync(0xffffffffu, x[a], own);
      if (m < total) {
        const uint32_t r = m - (o_inc - o_ic);
        int na[3], za[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
          za[a] = (int)((o_opts >> (2 * a)) & 1u);
          na[a] = 1 + za[a] + (int)((o_opts >> (2 * a + 1)) & 1u);
        }
        const uint32_t zero = (uint32_t)((za[2] * na[1] + za[1]) * na[0] + za[0]);
        const uint32_t e = r + (r >= zero ? 1u : 0u);
        const int sh[3] = {(int)(e % (uint32_t)na[0]) - za[0],
                           (int)((e / (uint32_t)na[0]) % (uint32_t)na[1]) - za[1],
                           (int)(e / (uint32_t)(na[0] * na[1])) - za[2]};
        const BoxDev &bx = boxes[o_b];
        double c[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
          c[a] = ox[a];
          if (sh[a] != 0) image_coord<PT>(bx.g, ox[a], a, sh[a], &c[a]);
        }
        const uint32_t q = o_q0 + r;
        if (q < np_cap) emit_one<PT>(bx.g, bx.top_base, k3all, q, c, (uint32_t)o_i, keys, vals, ppos);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Runs of equal fine-cell keys.
// ---------------------------------------------------------------------------

// Fine cell of a stored processed particle, packed gx | gy << 21 | gz << 42,
// and its box: the stored coordinates are those its sort key was computed
// from, so (box, fine cell) is that key's exactly.
template <class PT>
__device__ __forceinline__ uint64_t stored_cell(const BoxDev *boxes, const uint64_t *s_base,
                                                int nbox, const SPos<PT> &sp, int *box) {
  const int b = nbox > 1 ? box_search(s_base, nbox, (uint64_t)sp.src) : 0;
  const Geom &g = boxes[b].g;
  const double c[3] = {as_d(sp.x), as_d(sp.y), as_d(sp.z)};
  uint64_t packed = 0;
#pragma unroll
  for (int a = 0; a < 3; a++)
    packed |= (uint64_t)fine_index(c[a], g.rmin[a], g.inv_h, g.G[a]) << (21 * a);
  *box = b;
  return packed;
}

// Cell-ordered positions, their packed fine cells (the sort leaves only the
// order) and run-start flags (a new (box, fine cell) pair) of the processed
// particles (their scan reads no more).  A warp takes two groups of 32 consecutive elements per step (w0 and
// w0 + stride), with both gathers in flight before either is used.  Lane l
// compares with lane l-1's cell; lane 0 recomputes its predecessor's.
template <class PT>
__global__ void __launch_bounds__(kT) k_gather_flags(const uint32_t *__restrict__ perm,
                                                     const SPos<PT> *__restrict__ ppos,
                                                     const BoxDev *__restrict__ boxes, int nbox,
                                                     SPos<PT> *__restrict__ spos,
                                                     uint64_t *__restrict__ cells,
                                                     uint32_t *__restrict__ flag,
                                                     const DevScal *__restrict__ sc) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  __shared__ uint64_t s_base[kMaxBoxes];
  load_bases(boxes, nbox, s_base, false);
  const int64_t np = sc->np;
  const int lane = threadIdx.x & 31;
  const int64_t st = gstride();
  for (int64_t w0 = gtid() - lane; w0 < np; w0 += 2 * st) {
    int64_t i[2] = {w0 + lane, w0 + st + lane};
    uint32_t pi[2] = {0u, 0u}, pp[2] = {0u, 0u};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (i[h] < np) pi[h] = perm[i[h]];
      if (lane == 0 && i[h] > 0 && i[h] < np) pp[h] = perm[i[h] - 1];
    }
    SPos<PT> sp[2], sq[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (i[h] < np) sp[h] = ppos[pi[h]];
      if (lane == 0 && i[h] > 0 && i[h] < np) sq[h] = ppos[pp[h]];
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      uint64_t cell = 0;
      int box = 0;
      if (i[h] < np) {
        spos[i[h]] = sp[h];
        cell = stored_cell<PT>(boxes, s_base, nbox, sp[h], &box);
        cells[i[h]] = cell;
      }
      uint64_t pcell = __shfl_up_sync(0xffffffffu, cell, 1);
      int pbox = __shfl_up_sync(0xffffffffu, box, 1);
      if (lane == 0 && i[h] > 0 && i[h] < np) pcell = stored_cell<PT>(boxes, s_base, nbox, sq[h], &pbox);
      if (i[h] < np) flag[i[h]] = (i[h] == 0 || cell != pcell || box != pbox) ? 1u : 0u;
    }
  }
}

__device__ __forceinline__ uint64_t top_of_run(const BoxDev &bx, uint64_t pg) {
  const Geom &g = bx.g;
  const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
  return bx.top_base +
         ((uint64_t)div_k(gz, g) * g.T[1] + (uint64_t)div_k(gy, g)) * g.T[0] + div_k(gx, g);
}

// Run of every processed particle, and per run its first particle, packed
// fine cell, box and initial parent (itself); the range of runs of every
// occupied top cell ([first, last + 1), written where the top cell changes
// between neighbouring particles; top_range starts zeroed).
template <class PT>
__global__ void __launch_bounds__(kT) k_runs(const uint64_t *__restrict__ cells,
                                             const uint32_t *__restrict__ flag,
                                             const uint32_t *__restrict__ run_scan,
                                             const SPos<PT> *__restrict__ spos,
                                             const BoxDev *__restrict__ boxes, int nbox,
                                             DevScal *sc,
                                             uint32_t *__restrict__ run_of,
                                             uint32_t *__restrict__ run_start,
                                             uint64_t *__restrict__ run_g,
                                             uint16_t *__restrict__ run_box,
                                             uint32_t *__restrict__ parent,
                                             uint32_t *__restrict__ top_range) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  __shared__ uint64_t s_base[kMaxBoxes];
  load_bases(boxes, nbox, s_base, false);
  const int64_t np = sc->np;
  const uint32_t R = sc->R;
  auto box_of = [&](int64_t i) {
    return nbox > 1 ? box_search(s_base, nbox, (uint64_t)spos[i].src) : 0;
  };
  for (int64_t i = gtid(); i < np; i += gstride()) {
    const uint32_t f = flag[i];
    const uint32_t rid = run_scan[i] + f - 1u;
    const bool last = i == np - 1 || flag[i + 1] != 0u;
    run_of[i] = rid;
    if (!f && !last) continue;
    const uint64_t c = cells[i];
    const int b = box_of(i);
    const uint64_t t = top_of_run(boxes[b], c);
    if (f) {
      run_start[rid] = (uint32_t)i;
      run_g[rid] = c;
      run_box[rid] = (uint16_t)b;
      parent[rid] = rid;
      if (i == 0 || top_of_run(boxes[box_of(i - 1)], cells[i - 1]) != t)
        top_range[2 * t] = rid;
    }
    if (last && (i == np - 1 || top_of_run(boxes[box_of(i + 1)], cells[i + 1]) != t))
      top_range[2 * t + 1] = rid + 1u;
    if (i == np - 1) run_start[R] = (uint32_t)np;
  }
}

// Grid cell and linking length of every processed particle (variable
// linking length runs only; boxes with a fixed length get cell 0 and their
// own l^2, which reproduces the fixed-length test).
template <class PT, bool FP32>
__global__ void __launch_bounds__(kT) k_varlink_recs(const SPos<PT> *__restrict__ spos,
                                                     const uint32_t *__restrict__ run_of,
                                                     const uint16_t *__restrict__ run_box,
                                                     const BoxDev *__restrict__ boxes,
                                                     const DevScal *__restrict__ sc,
                                                     VLRec<FP32> *__restrict__ svl) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const int64_t np = sc->np;
  for (int64_t i = gtid(); i < np; i += gstride()) {
    const Geom &g = boxes[run_box[run_of[i]]].g;
    VLRec<FP32> v;
    v.rkey = 0;
    v.lsq = g.linksq;
    if (g.varlink) {
      const SPos<PT> p = spos[i];
      v.rkey = ref_key(g, (double)p.x, (double)p.y, (double)p.z);
      v.lsq = ref_cell_linksq(g, v.rkey);
    }
    svl[i] = v;
  }
}

// Dense top cells with more fine cells than this are joined by a whole CTA,
// the others by one warp each.
constexpr uint32_t kBigTop = 64;

// Warp-aggregated slot from a counter for the lanes with `pick` set: one
// atomic per warp, the lanes in lane order after the returned base.
__device__ __forceinline__ uint32_t warp_slot(bool pick, uint32_t *counter) {
  const uint32_t m = __ballot_sync(0xffffffffu, pick);
  if (m == 0) return 0u;
  const int lane = threadIdx.x & 31, first = __ffs(m) - 1;
  uint32_t base = 0;
  if (lane == first) base = atomicAdd(counter, (uint32_t)__popc(m));
  base = __shfl_sync(0xffffffffu, base, first);
  return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

// Dense top cells (more than dense_min fine cells), one thread per fine
// cell, acting at each top cell's first: a slot from a counter (the order of
// the slots does not matter), the top cell's slot and fine-cell range, and
// the big ones' slots listed in `big`.  Past nd_cap a dense top cell gets no
// slot and is scanned instead (slower but exact), and the overflow bit asks
// the plan for more slots next time.
__global__ void __launch_bounds__(kT) k_dense_pick(const uint64_t *__restrict__ run_g,
                                                   const uint16_t *__restrict__ run_box,
                                                   const BoxDev *__restrict__ boxes,
                                                   DevScal *sc,
                                                   const uint2 *__restrict__ top_range,
                                                   uint32_t dense_min, uint32_t nd_cap,
                                                   uint32_t *__restrict__ top_slot,
                                                   uint2 *__restrict__ dense_range,
                                                   uint32_t *__restrict__ big) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const uint32_t R = sc->R;
  const int lane = threadIdx.x & 31;
  for (int64_t r0 = gtid() - lane; r0 < (int64_t)R; r0 += gstride()) {
    const int64_t r = r0 + lane;
    bool pick = false;
    uint64_t t = 0;
    uint2 tr = make_uint2(0u, 0u);
    if (r < (int64_t)R) {
      t = top_of_run(boxes[run_box[r]], run_g[r]);
      tr = top_range[t];
      pick = tr.x == (uint32_t)r && tr.y - tr.x > dense_min;
    }
    const uint32_t slot = warp_slot(pick, &sc->nd);
    if (!pick) continue;
    if (slot < nd_cap) {
      top_slot[t] = slot;
      dense_range[slot] = tr;
      if (tr.y - tr.x > kBigTop) big[atomicAdd(&sc->nbig, 1u)] = slot;
    } else {
      atomicOr(&sc->overflow, 2u);
    }
  }
}


// ---------------------------------------------------------------------------
// Befriending.
// ---------------------------------------------------------------------------

// The reference's pair predicate (FOF.c:351-357), FP64 or FP32 + band recheck.
// With VL (variable linking length) the pair's l^2 or band comes from the
// lower of the two particles' grid cells, and particles of cells that are
// not neighbours are never linked; va/vb are ignored otherwise.
template <class PT, bool FP32, bool VL>
__device__ __forceinline__ bool linked(const SPos<PT> &p, const SPos<PT> &q, const Geom &g,
                                       const VLRec<FP32> &va, const VLRec<FP32> &vb,
                                       unsigned long long &rechecks) {
  float t_lo = g.t_lo, t_hi = g.t_hi;
  double lsq = g.linksq;
  if constexpr (VL) {
    if (!ref_neighbours(va.rkey, vb.rkey)) return false;
    lsq = (va.rkey <= vb.rkey ? va : vb).lsq;
    if constexpr (FP32) vl_band(lsq, sizeof(PT) == 4 ? 4 : 8, &t_lo, &t_hi);
  }
  double dx, dy, dz;
  if constexpr (sizeof(PT) == 4) {
    const float fx = __fsub_rn(p.x, q.x), fy = __fsub_rn(p.y, q.y), fz = __fsub_rn(p.z, q.z);
    if constexpr (FP32) {
      const float d2 = __fmaf_rn(fz, fz, __fmaf_rn(fy, fy, __fmul_rn(fx, fx)));
      if (d2 < t_lo) return true;
      if (d2 > t_hi) return false;
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
      if (d2 < t_lo) return true;
      if (d2 > t_hi) return false;
      rechecks++;
    }
  }
  const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return !(d2 > lsq);
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

// Per-thread tallies of the befriending kernels, flushed once per warp.
struct BfStats {
  unsigned long long tests = 0, rechecks = 0, cand = 0, skips = 0, unions = 0, steps = 0;
  unsigned long long scan = 0, window = 0;

  __device__ void flush(Counters *ctr) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      tests += __shfl_down_sync(0xffffffffu, tests, d);
      rechecks += __shfl_down_sync(0xffffffffu, rechecks, d);
      cand += __shfl_down_sync(0xffffffffu, cand, d);
      skips += __shfl_down_sync(0xffffffffu, skips, d);
      unions += __shfl_down_sync(0xffffffffu, unions, d);
      steps += __shfl_down_sync(0xffffffffu, steps, d);
      scan += __shfl_down_sync(0xffffffffu, scan, d);
      window += __shfl_down_sync(0xffffffffu, window, d);
    }
    if ((threadIdx.x & 31) == 0) {
      if (tests) atomicAdd(&ctr->pair_tests, tests);
      if (rechecks) atomicAdd(&ctr->rechecks, rechecks);
      if (cand) atomicAdd(&ctr->cand_pairs, cand);
      if (skips) atomicAdd(&ctr->root_skips, skips);
      if (unions) atomicAdd(&ctr->unions, unions);
      if (steps) atomicAdd(&ctr->find_steps, steps);
      if (scan) atomicAdd(&ctr->scan_iters, scan);
      if (window) atomicAdd(&ctr->window_iters, window);
    }
  }
};

// Whether any particle of fine cell a (particles [sa, ea), fine coordinates
// ax, ay, az) is linked to any particle of fine cell b (fine coordinates bx,
// by, bz).  The loop runs over the cell with fewer particles, and each of
// its particles farther than the linking length from the other cell's box
// is skipped; the pair predicate is symmetric (the difference of a pair
// only changes sign, and a variable length comes from the lower of the two
// grid cells), so the orientation does not change the answer.  Every 16
// particles, `apart()` is asked whether a and b are still in different
// components (another thread may have joined them meanwhile); if not, the
// search stops and reports no link, which is then harmless.
template <class PT, bool FP32, bool VL, class Apart>
__device__ __forceinline__ bool cells_linked(const Geom &g, int ax, int ay, int az, uint32_t sa,
                                             uint32_t ea, uint32_t b, int bx, int by, int bz,
                                             const uint32_t *__restrict__ run_start,
                                             const SPos<PT> *__restrict__ spos,
                                             const VLRec<FP32> *__restrict__ svl, BfStats &st,
                                             Apart apart) {
  uint32_t sb = __ldg(run_start + b), eb = __ldg(run_start + b + 1);
  if (eb - sb < ea - sa) {
    uint32_t t = sa;
    sa = sb;
    sb = t;
    t = ea;
    ea = eb;
    eb = t;
    bx = ax;
    by = ay;
    bz = az;
  }
  for (uint32_t i = sa; i < ea; i++) {
    if (((i - sa) & 15) == 15 && !apart()) return false;
    const SPos<PT> p = spos[i];
    if (box_dist2(g, (double)p.x, (double)p.y, (double)p.z, bx, by, bz) > g.prune_sq) continue;
    VLRec<FP32> va{};
    if constexpr (VL) va = svl[i];
    for (uint32_t j = sb; j < eb; j++) {
      st.tests++;
      VLRec<FP32> vb{};
      if constexpr (VL) vb = svl[j];
      if (linked<PT, FP32, VL>(p, spos[j], g, va, vb, st.rechecks)) return true;
    }
  }
  return false;
}

// Link fine cells a and b if any pair of their particles is linked.  The
// cells are internally connected, so one linked pair joins them entirely.
// `ra` caches a root of a's component: it may be stale (a root that was hooked
// since), but it stays in a's component, so "b reaches ra" still proves that
// a and b are already joined.
template <class PT, bool FP32, bool VL>
__device__ __forceinline__ void try_link(const Geom &g, uint32_t a, int ax, int ay, int az,
                                         uint32_t &ra, uint32_t b,
                                         int bx, int by, int bz, uint32_t sa, uint32_t ea,
                                         const uint32_t *__restrict__ run_start,
                                         const SPos<PT> *__restrict__ spos,
                                         const VLRec<FP32> *__restrict__ svl, uint32_t *parent,
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
  if (cells_linked<PT, FP32, VL>(g, ax, ay, az, sa, ea, b, bx, by, bz, run_start, spos, svl, st,
                                 apart)) {
    uf_union(parent, ra, rb, ctr, g.union_cap);
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

// Returns whether this call joined two components.
__device__ __forceinline__ bool lunion(uint32_t *lp, uint32_t a, uint32_t b, Counters *ctr,
                                       uint32_t cap) {
  for (uint32_t it = 0; it < cap; it++) {
    a = lfind(lp, a);
    b = lfind(lp, b);
    if (a == b) return false;
    if (a < b) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    const uint32_t old = atomicCAS(lp + a, a, b);
    if (old == a) return true;
    a = old;
  }
  atomicAdd(&ctr->uf_giveups, 1u);
  return false;
}

// Bits lo..hi (0 <= lo <= hi <= 31) set.
__device__ __forceinline__ uint32_t bit_span(int lo, int hi) {
  return (hi - lo == 31 ? 0xffffffffu : ((1u << (hi - lo + 1)) - 1u)) << lo;
}

// Dense top cells: the fine-cell pairs inside a top cell are joined with a
// union-find in shared memory, near pairs before far ones; then every fine
// cell is joined to its local root in the global union-find (a
// compare-and-swap of its own parent when nothing else has hooked it, a
// union otherwise: the sparse kernel runs at the same time).  Links that cross the top
// cell's faces are left to the global passes.  The occupied fine cells of
// the top cell are first marked in bit rows (bit x of rows[z k + y]), so a
// cell visits only the occupied cells of its forward window, a row at a
// time, and finds their local indices from the rows' prefix counts.  `tid`/`nt` number the
// threads that share the top cell and `sync` is their barrier; `lpar` holds
// k3all parents followed by the k^2 rows and their k^2 prefix counts.
template <class PT, bool FP32, bool VL, class Sync>
__device__ __forceinline__ void dense_top(uint32_t slot, uint32_t *lpar, uint32_t tid,
                                          uint32_t nt, Sync sync, const BoxDev *boxes,
                                          const uint16_t *run_box, uint64_t k3all,
                                          const uint32_t *run_start, const uint64_t *run_g,
                                          const uint2 *dense_range, uint32_t *grows,
                                          uint32_t kk, const SPos<PT> *spos,
                                          const VLRec<FP32> *svl, uint32_t *parent,
                                          Counters *ctr, BfStats &st) {
  const uint2 fr = dense_range[slot];
  const uint32_t f = fr.x, n = fr.y - fr.x;
  const Geom &g = boxes[run_box[f]].g;
  const int k = g.k, W = g.W;
  const uint32_t nrow = (uint32_t)(k * k);
  uint32_t *rows = lpar + k3all;   // occupancy bits of each (z, y) row
  uint32_t *pref = rows + nrow;    // occupied fine cells before each row
  // components left: once one is left, every remaining candidate is joined
  volatile uint32_t *ncomp = lpar + k3all + 2 * kk;
  if (tid == 0) *ncomp = n;
  for (uint32_t i = tid; i < n; i += nt) lpar[i] = i;
  for (uint32_t j = tid; j < nrow; j += nt) rows[j] = 0u;
  sync();
  for (uint32_t i = tid; i < n; i += nt) {
    const uint64_t pg = run_g[f + i];
    const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
    atomicOr(rows + (gz - div_k(gz, g) * k) * k + (gy - div_k(gy, g) * k),
             1u << (gx - div_k(gx, g) * k));
  }
  sync();
  if (tid < 32) {
    // the top cell's fine cells are in sub-cell order, so a cell's local
    // index is the number of occupied cells in the rows before it plus those
    // before it in its row: prefix of the row populations, one warp
    const uint32_t per = (nrow + 31) / 32, j0 = tid * per, j1 = min(j0 + per, nrow);
    uint32_t sum = 0;
    for (uint32_t j = j0; j < j1; j++) sum += __popc(rows[j]);
    uint32_t inc = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, d);
      if (tid >= (uint32_t)d) inc += t;
    }
    uint32_t acc = inc - sum;
    for (uint32_t j = j0; j < j1; j++) {
      pref[j] = acc;
      acc += __popc(rows[j]);
    }
  }
  sync();
  for (int pass = 0; pass < 2; pass++) {
    for (uint32_t i = tid; i < n; i += nt) {
      if (*ncomp == 1) break;
      const uint32_t a = f + i;
      const uint64_t pg = run_g[a];
      const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
      const int sx = gx - div_k(gx, g) * k, sy = gy - div_k(gy, g) * k, sz = gz - div_k(gz, g) * k;
      const uint32_t sa = run_start[a], ea = run_start[a + 1];
      // columns within reach, and the near ones (|dx| <= 1)
      const uint32_t reach = bit_span(max(sx - W, 0), min(sx + W, k - 1));
      const uint32_t near = bit_span(max(sx - 1, 0), min(sx + 1, k - 1));
      const uint32_t after = sx == 31 ? 0u : (0xffffffffu << (sx + 1));
      uint32_t ri = lfind(lpar, i);  // may go stale: re-found before a pair test
      for (int dz = 0; dz <= W && sz + dz < k; dz++)
        for (int dy = (dz == 0 ? 0 : -W); dy <= W; dy++) {
          const int ty = sy + dy;
          if (ty < 0 || ty >= k) continue;
          if (*ncomp == 1) break;
          const int rc = max(abs(dy), dz);  // the row's distance in y and z
          uint32_t m;
          if (pass == 0) m = rc <= 1 ? near : 0u;       // Chebyshev distance <= 1
          else m = rc <= 1 ? (reach & ~near) : reach;   // Chebyshev distance >= 2
          if (dz == 0 && dy == 0) m &= after;           // forward only in a's own row
          const int tz = sz + dz;
          const uint32_t row = (uint32_t)(tz * k + ty);
          const uint32_t occ = rows[row];
          uint32_t bits = occ & m;
          while (bits) {
            const int tx = __ffs(bits) - 1;
            bits &= bits - 1u;
            const uint32_t lj = pref[row] + __popc(occ & ((1u << tx) - 1u));
            st.cand++;
            const uint32_t rj = lfind(lpar, lj);
            if (rj == ri || rj == (ri = lfind(lpar, i))) {
              st.skips++;
              continue;
            }
            auto apart = [&]() { return lfind(lpar, i) != lfind(lpar, lj); };
            if (cells_linked<PT, FP32, VL>(g, gx, gy, gz, sa, ea, f + lj, gx + (tx - sx), gy + dy,
                                           gz + dz, run_start, spos, svl, st, apart)) {
              if (lunion(lpar, ri, rj, ctr, g.union_cap))
                atomicSub(const_cast<uint32_t *>(ncomp), 1u);
              st.unions++;
            }
          }
        }
    }
    sync();
  }
  // joined to its local root through the global union-find: the sparse
  // kernel runs at the same time and may have hooked a cell of this top cell
  for (uint32_t i = tid; i < n; i += nt) {
    const uint32_t r = f + lfind(lpar, i);
    if (r != f + i && atomicCAS(parent + f + i, f + i, r) != f + i)
      uf_union(parent, f + i, r, ctr, g.union_cap);
  }
  // rows and prefixes stay for the warp path, which looks up this top
  // cell's fine cells from its neighbours
  uint32_t *gr = grows + (uint64_t)slot * 2 * kk;
  for (uint32_t j = tid; j < nrow; j += nt) {
    gr[j] = rows[j];
    gr[kk + j] = pref[j];
  }
  sync();
}

// The dense top cells.  The big ones (more than kBigTop fine cells, listed
// in `big`) go first, one per CTA, so that the largest, which bound the
// kernel's length, start early and have many threads; then each warp takes
// the small ones one at a time, with its own slice of `lstride` words of
// shared memory (parents and bit rows).  Both kinds are taken from atomic counters: their sizes
// differ widely.
template <class PT, bool FP32, bool VL>
__global__ void __launch_bounds__(128) k_befriend_dense(
    const BoxDev *__restrict__ boxes, const uint16_t *__restrict__ run_box, uint64_t k3all,
    const uint32_t *__restrict__ run_start, const uint64_t *__restrict__ run_g,
    const uint2 *__restrict__ dense_range, const uint32_t *__restrict__ big, DevScal *sc,
    uint32_t nd_cap, uint32_t *__restrict__ grows, uint32_t kk,
    const SPos<PT> *__restrict__ spos, const VLRec<FP32> *__restrict__ svl, uint32_t *parent,
    Counters *ctr, uint32_t lstride) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  extern __shared__ uint32_t smem[];
  __shared__ uint32_t s_slot;
  const uint32_t nd = min(sc->nd, nd_cap), nbig = sc->nbig;
  BfStats st;
  auto cta_sync = []() { __syncthreads(); };
  while (true) {
    if (threadIdx.x == 0) {
      const uint32_t b = atomicAdd(&sc->next_big, 1u);
      s_slot = b < nbig ? big[b] : kNone;
    }
    __syncthreads();
    const uint32_t slot = s_slot;
    __syncthreads();
    if (slot == kNone) break;
    dense_top<PT, FP32, VL>(slot, smem, threadIdx.x, blockDim.x, cta_sync, boxes, run_box,
                            k3all, run_start, run_g, dense_range, grows, kk, spos, svl, parent,
                            ctr, st);
  }
  const uint32_t lane = threadIdx.x & 31;
  uint32_t *lpar = smem + (size_t)(threadIdx.x >> 5) * lstride;
  auto warp_sync = []() { __syncwarp(); };
  while (true) {
    uint32_t slot = 0;
    if (lane == 0) slot = atomicAdd(&sc->next_dense, 1u);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    if (slot >= nd) break;
    const uint2 fr = dense_range[slot];
    if (fr.y - fr.x > kBigTop) continue;
    dense_top<PT, FP32, VL>(slot, lpar, lane, 32, warp_sync, boxes, run_box, k3all, run_start,
                            run_g, dense_range, grows, kk, spos, svl, parent, ctr, st);
  }
  st.flush(ctr);
}

// Whether fine cell a's neighbour top cell in direction o lies within W fine
// cells of a (s = a's fine coordinate inside its top cell).
__device__ __forceinline__ bool reaches(int s, int o, int k, int W) {
  return o == 0 || (o > 0 ? s >= k - W : s <= W - 1);
}

// Candidates of fine cell a are the fine cells b > a (key order, so each
// unordered pair is visited once) within W fine cells on every axis; they
// live in a's top cell (after a) and the 13 forward top cells.
//
// Fast path, one thread per fine cell: the ranges of the top cells a can
// reach are loaded at once; when none holds more than kSimple candidate cells
// (the common case away from clumps), the first of each is loaded at once too
// and the cell is finished in two L2 round trips.  Other cells are queued for
// the warp path below.
constexpr uint32_t kSimple = 2;  // two slot bits per range below
constexpr uint32_t kSimpleChunk = 1024;  // fine cells per grab of a CTA

template <class PT, bool FP32, bool VL>
__global__ void __launch_bounds__(kT, 5) k_befriend_simple(
    const BoxDev *__restrict__ boxes, const uint16_t *__restrict__ run_box,
    const uint32_t *__restrict__ run_start, const uint64_t *__restrict__ run_g, DevScal *sc,
    const uint2 *__restrict__ top_range,
    const uint32_t *__restrict__ top_slot, const SPos<PT> *__restrict__ spos,
    const VLRec<FP32> *__restrict__ svl, uint32_t *parent, uint32_t *__restrict__ queue,
    Counters *ctr) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const uint32_t R = sc->R;
  const int lane = threadIdx.x & 31;
  __shared__ uint32_t s_base;
  BfStats st;
  // CTAs take chunks of consecutive fine cells from a counter: the work per
  // cell varies a lot across the box (clumps, queued cells), and a static
  // share would leave the CTAs of the busy regions running alone at the end
  while (true) {
    if (threadIdx.x == 0) s_base = atomicAdd(&sc->next_simple, kSimpleChunk);
    __syncthreads();
    const uint32_t base = s_base;
    __syncthreads();
    if (base >= R) break;
    const uint32_t end = min(base + kSimpleChunk, R);
    for (uint32_t a = base + threadIdx.x; a < end; a += blockDim.x) {
    const BoxDev &bx = boxes[run_box[a]];
    const Geom &g = bx.g;
    const int k = g.k, W = g.W;
    const uint64_t pg = run_g[a];
    const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
    const int tx = div_k(gx, g), ty = div_k(gy, g), tz = div_k(gz, g);
    const int sx = gx - tx * k, sy = gy - ty * k, sz = gz - tz * k;
    uint32_t R0[14], NN[14];
#pragma unroll
    for (int nb = 0; nb < 14; nb++) {
      const int ux = tx + kFwd[nb][0], uy = ty + kFwd[nb][1], uz = tz + kFwd[nb][2];
      // a top cell more than W fine cells away from a is skipped without a load
      const bool in = !(ux < 0 || uy < 0 || ux >= g.T[0] || uy >= g.T[1] || uz >= g.T[2]) &&
                      reaches(sx, kFwd[nb][0], k, W) && reaches(sy, kFwd[nb][1], k, W) &&
                      reaches(sz, kFwd[nb][2], k, W);
      const uint64_t tb = in ? bx.top_base + ((uint64_t)uz * g.T[1] + uy) * g.T[0] + ux : 0;
      const uint2 tr = in ? top_range[tb] : make_uint2(0u, 0u);
      const uint32_t f = tr.x, e = tr.y;
      R0[nb] = nb == 0 ? a + 1 : f;
      NN[nb] = e > R0[nb] ? e - R0[nb] : 0u;
      // pairs inside a dense top cell are joined by k_befriend_dense
      if (nb == 0 && in && top_slot[tb] != kNone) NN[nb] = 0u;
    }
    bool simple = true;
#pragma unroll
    for (int nb = 0; nb < 14; nb++) simple &= NN[nb] <= kSimple;
    const unsigned active = __activemask();
    const unsigned qmask = __ballot_sync(active, !simple);
    if (qmask) {
      const int leader = __ffs(qmask) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(&sc->qcount, (uint32_t)__popc(qmask));
      base = __shfl_sync(active, base, leader);
      if (!simple) queue[base + __popc(qmask & ((1u << lane) - 1u))] = a;
    }
    if (!simple) continue;
    // candidate slots: bit 2 nb + q stands for fine cell R0[nb] + q.  The
    // first fine cell of every range is loaded at once and dropped here when
    // out of reach; the slots left are visited from one call site below (a
    // single inlined copy of the link test keeps the kernel's code small)
    uint32_t m = 0;
#pragma unroll
    for (int nb = 0; nb < 14; nb++) {
      if (NN[nb] == 0) continue;
      st.scan += NN[nb];
      const uint64_t qg = run_g[R0[nb]];
      const int bx2 = (int)(qg & kM21), by2 = (int)((qg >> 21) & kM21), bz2 = (int)(qg >> 42);
      if (max(abs(bx2 - gx), max(abs(by2 - gy), abs(bz2 - gz))) <= W) m |= 1u << (2 * nb);
      if (NN[nb] > 1) m |= 2u << (2 * nb);
    }
    uint32_t ra = 0xffffffffu, sa = 0, ea = 0;
    while (m) {
      const int bit = __ffs(m) - 1;
      m &= m - 1;
      const int nb = bit >> 1;
      uint32_t r = 0;
#pragma unroll
      for (int t = 0; t < 14; t++) r = t == nb ? R0[t] : r;
      r += (uint32_t)(bit & 1);
      const uint64_t qg = run_g[r];  // L1 hit for the first cell of a range
      const int bx2 = (int)(qg & kM21), by2 = (int)((qg >> 21) & kM21), bz2 = (int)(qg >> 42);
      if ((bit & 1) && max(abs(bx2 - gx), max(abs(by2 - gy), abs(bz2 - gz))) > W) continue;
      if (ra == 0xffffffffu) {
        ra = __ldcg(parent + a);
        sa = run_start[a];
        ea = run_start[a + 1];
      }
      try_link<PT, FP32, VL>(g, a, gx, gy, gz, ra, r, bx2, by2, bz2, sa, ea, run_start, spos, svl, parent,
                             ctr, st);
    }
    }
  }
  st.flush(ctr);
}

// Warp path, one warp per queued fine cell a.  Lanes 0..13 fetch the 14
// top-cell ranges at once; the candidate slots of all 14 (fine cells of small
// top cells, window slots of dense ones, found through their occupancy rows)
// are then flattened and taken 32 at a time, so a cell costs a few L2 round
// trips instead of one per slot.  Warps take cells from an atomic counter as they finish, so a few
// expensive cells do not hold back a whole static share.  PHASE 0 visits the
// candidates within one fine cell, PHASE 1 the farther ones, so that a dense
// neighbourhood is joined (and compressed) before its far pairs are tried and
// most of those become root skips.
template <class PT, bool FP32, bool VL, int PHASE>
__global__ void __launch_bounds__(kT, 4) k_befriend(
    const BoxDev *__restrict__ boxes, const uint16_t *__restrict__ run_box, uint64_t k3all,
    const uint32_t *__restrict__ run_start, const uint64_t *__restrict__ run_g,
    const uint32_t *__restrict__ queue, DevScal *sc, const uint2 *__restrict__ top_range,
    const uint32_t *__restrict__ top_slot,
    const uint32_t *__restrict__ grows, uint32_t kk, const SPos<PT> *__restrict__ spos,
    const VLRec<FP32> *__restrict__ svl, uint32_t *parent, Counters *ctr) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const uint32_t NQ = sc->qcount;
  uint32_t *next = PHASE == 0 ? &sc->next0 : &sc->next1;
  const int lane = threadIdx.x & 31;
  BfStats st;
  while (true) {
    uint32_t qi = 0;
    if (lane == 0) qi = atomicAdd(next, 1u);
    qi = __shfl_sync(0xffffffffu, qi, 0);
    if (qi >= NQ) break;
    const uint32_t a = queue[qi];
    const BoxDev &bx = boxes[run_box[a]];
    const Geom &g = bx.g;
    const int k = g.k, W = g.W;
    const uint64_t pg = run_g[a];
    const int gx = (int)(pg & kM21), gy = (int)((pg >> 21) & kM21), gz = (int)(pg >> 42);
    const int tx = div_k(gx, g), ty = div_k(gy, g), tz = div_k(gz, g);
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
        const uint64_t tb = bx.top_base + ((uint64_t)uz * g.T[1] + uy) * g.T[0] + ux;
        const uint2 tr = top_range[tb];
        const uint32_t f = tr.x, e = tr.y;
        const uint32_t slot = top_slot[tb];
        r0 = lane == 0 ? a + 1 : f;
        // pairs inside a dense top cell are joined by k_befriend_dense
        if (lane == 0 && slot != kNone) r0 = e;
        if (r0 < e) {
          if (slot == kNone) {
            nsparse = e - r0;
          } else {
            x0 = max(gx - W, ux * k);
            const int x1 = min(gx + W, ux * k + k - 1);
            y0 = max(gy - W, uy * k);
            const int y1 = min(gy + W, uy * k + k - 1);
            z0 = max(gz - W, uz * k);
            const int z1 = min(gz + W, uz * k + k - 1);
            if (x1 >= x0 && y1 >= y0 && z1 >= z0) {
              nx = x1 - x0 + 1;
              ny = y1 - y0 + 1;
              nslots = (uint32_t)(nx * ny * (z1 - z0 + 1));
              mapbase = slot;
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
      int bx2, by2, bz2;
      if (off < l_ns) {
        st.scan++;
        r = l_r0 + off;
        const uint64_t qg = run_g[r];
        bx2 = (int)(qg & kM21);
        by2 = (int)((qg >> 21) & kM21);
        bz2 = (int)(qg >> 42);
        if (max(abs(bx2 - gx), max(abs(by2 - gy), abs(bz2 - gz))) > W) continue;
      } else {
        st.window++;
        const uint32_t sl = off - l_ns;
        bx2 = l_x0 + (int)(sl % (uint32_t)l_nx);
        by2 = l_y0 + (int)((sl / (uint32_t)l_nx) % (uint32_t)l_ny);
        bz2 = l_z0 + (int)(sl / (uint32_t)(l_nx * l_ny));
        // a slot of the other phase is dropped before its row is read
        const int cheb_s = max(abs(bx2 - gx), max(abs(by2 - gy), abs(bz2 - gz)));
        if ((PHASE == 0 && cheb_s > 1) || (PHASE == 1 && cheb_s <= 1)) continue;
        // occupancy bit of the slot's fine cell, then its index from the
        // top cell's row prefix (fine cells are in sub-cell order)
        const uint32_t *gr = grows + (uint64_t)l_map * 2 * kk;
        const uint32_t row = (uint32_t)((bz2 - l_oz) * k + (by2 - l_oy));
        const uint32_t occ = gr[row];
        const int cx = bx2 - l_ox;
        if (!((occ >> cx) & 1u)) continue;
        r = l_r0 + gr[kk + row] + __popc(occ & ((1u << cx) - 1u));
      }
      const int cheb = max(abs(bx2 - gx), max(abs(by2 - gy), abs(bz2 - gz)));
      if ((PHASE == 0 && cheb > 1) || (PHASE == 1 && cheb <= 1)) continue;
      try_link<PT, FP32, VL>(g, a, gx, gy, gz, ra, r, bx2, by2, bz2, sa, ea, run_start, spos, svl, parent, ctr,
                             st);
    }
  }
  st.flush(ctr);
}

__global__ void __launch_bounds__(kT) k_compress(uint32_t *parent,
                                                 const DevScal *__restrict__ sc) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const uint32_t R = sc->R;
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
                                                    const uint32_t *__restrict__ perm,
                                                    const DevScal *__restrict__ sc,
                                                    uint32_t *__restrict__ count,
                                                    uint32_t *__restrict__ head) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const int64_t np = sc->np;
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

// Subsampling (FOF.c:205-284): every original particle inside its box's
// domain ([lo, hi) per axis, [lo, hi] on the axes of `closed`) is kept when its uniform is
// below its group's rate -- samp_in for groups of at least Nphalomin
// processed particles (FOF.c:202), samp_out for the others.  The uniform is
// the top 53 bits of SplitMix64's output mix (Steele, Lea & Flood 2014) of
// key ^ (seed * 0xD1B54A32D192ED03), key = the particle's ID or its input
// index, so a particle's draw depends on nothing but the seed and itself.
__device__ __forceinline__ double sample_uniform(uint64_t seed, uint64_t key) {
  uint64_t z = key ^ (seed * 0xD1B54A32D192ED03ull);
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * 0x1.0p-53;
}

template <class PT>
__global__ void __launch_bounds__(kT) k_subsample(
    const uint32_t *__restrict__ run_of, const uint32_t *__restrict__ parent,
    const uint32_t *__restrict__ count, const uint32_t *__restrict__ perm,
    const SPos<PT> *__restrict__ spos, const uint16_t *__restrict__ run_box,
    const BoxDev *__restrict__ boxes, const uint32_t *__restrict__ boxd, int nbox,
    const DevScal *__restrict__ sc, const uint64_t *__restrict__ ids, double samp_in,
    double samp_out, uint64_t seed, int closed, uint8_t *__restrict__ samp) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const int64_t np = sc->np;
  for (int64_t i = gtid(); i < np; i += gstride()) {
    const uint32_t run = run_of[i];
    const int b = run_box[run];
    if (perm[i] - boxd[4 * nbox + b] >= boxd[2 * nbox + b]) continue;  // an image
    const Geom &g = boxes[b].g;
    const SPos<PT> sp = spos[i];
    const double x[3] = {as_d(sp.x), as_d(sp.y), as_d(sp.z)};
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; a++)
      inside &= x[a] >= g.lo[a] && (((closed >> a) & 1) ? x[a] <= g.hi[a] : x[a] < g.hi[a]);
    if (!inside) continue;
    const bool in = !((double)count[parent[run]] < g.nphalomin);
    const double rate = in ? samp_in : samp_out;
    if (!(rate > 0.0)) continue;
    const uint64_t key = ids ? ids[sp.src] : (uint64_t)sp.src;
    if (sample_uniform(seed, key) < rate) samp[sp.src] = in ? 1 : 2;
  }
}

// Candidate halos: roots of at least Nphalomin members (FOF.c:202), each
// given an index from a counter (the catalog is put in head order later, so
// the candidates' order does not matter); counts the roots (groups).
__global__ void __launch_bounds__(kT) k_cand_pick(const uint32_t *__restrict__ parent,
                                                  const uint32_t *__restrict__ count,
                                                  const uint16_t *__restrict__ run_box,
                                                  const BoxDev *__restrict__ boxes,
                                                  DevScal *sc,
                                                  uint32_t *__restrict__ cand_of_root,
                                                  uint32_t *__restrict__ cand_root,
                                                  unsigned long long *ngroups) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const uint32_t R = sc->R;
  const int lane = threadIdx.x & 31;
  unsigned long long roots = 0;
  for (int64_t r0 = gtid() - lane; r0 < (int64_t)R; r0 += gstride()) {
    const int64_t r = r0 + lane;
    bool cand = false;
    if (r < (int64_t)R) {
      const bool root = parent[r] == (uint32_t)r;
      roots += root;
      cand = root && !((double)count[r] < boxes[run_box[r]].g.nphalomin);
    }
    const uint32_t ci = warp_slot(cand, &sc->nc);
    if (cand) {
      cand_of_root[r] = ci;
      cand_root[ci] = (uint32_t)r;
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) roots += __shfl_down_sync(0xffffffffu, roots, d);
  if (lane == 0 && roots) atomicAdd(ngroups, roots);
}

// Property sums per candidate halo, in double as Output_Halos does
// (FOF.c:806-832): 6 first moments, then 6 position and 6 velocity second
// moments when INERTIA / DISPERSION are asked for.
template <class PT, int NS>
__global__ void __launch_bounds__(kT) k_group_sums(
    const uint32_t *__restrict__ run_of, const uint32_t *__restrict__ parent,
    const uint32_t *__restrict__ cand_of_root, const uint16_t *__restrict__ run_box,
    const BoxDev *__restrict__ boxes, const SPos<PT> *__restrict__ spos,
    const DevScal *__restrict__ sc, int props, double *__restrict__ sums,
    uint32_t *__restrict__ warn) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const int64_t np = sc->np;
  const int64_t n_iter = (np + 31) / 32 * 32;
  for (int64_t i = gtid(); i < n_iter; i += gstride()) {
    uint32_t ci = kNone;
    double v[NS];
#pragma unroll
    for (int c = 0; c < NS; c++) v[c] = 0.0;
    if (i < np) {
      const uint32_t run = run_of[i];
      ci = cand_of_root[parent[run]];
      if (ci != kNone) {
        const BoxDev &bx = boxes[run_box[run]];
        const Geom &g = bx.g;
        const SPos<PT> p = spos[i];
        const double x = (double)p.x, y = (double)p.y, z = (double)p.z;
        const uint64_t li = 3 * ((uint64_t)p.src - bx.in_base);
        double vx, vy, vz;
        if (bx.vel_f64) {
          const double *vel = static_cast<const double *>(bx.vel);
          vx = vel[li]; vy = vel[li + 1]; vz = vel[li + 2];
        } else {
          const float *vel = static_cast<const float *>(bx.vel);
          vx = (double)vel[li]; vy = (double)vel[li + 1]; vz = (double)vel[li + 2];
        }
        v[0] = x; v[1] = y; v[2] = z; v[3] = vx; v[4] = vy; v[5] = vz;
        if constexpr (NS >= 12) {
          if (props & 1) {
            v[6] = __dmul_rn(x, x); v[7] = __dmul_rn(y, y); v[8] = __dmul_rn(z, z);
            v[9] = __dmul_rn(x, y); v[10] = __dmul_rn(x, z); v[11] = __dmul_rn(y, z);
          }
        }
        if constexpr (NS >= 18) {
          v[12] = __dmul_rn(vx, vx); v[13] = __dmul_rn(vy, vy); v[14] = __dmul_rn(vz, vz);
          v[15] = __dmul_rn(vx, vy); v[16] = __dmul_rn(vx, vz); v[17] = __dmul_rn(vy, vz);
        } else if constexpr (NS >= 12) {
          if (!(props & 1)) {
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
// inside [lo, hi) on every axis.  An owned candidate is listed with its head
// as the key of the catalog's sort (from a counter: the sort by head fixes
// the order).
template <int NS>
__global__ void __launch_bounds__(kT) k_own_pick(const double *__restrict__ sums,
                                                 const uint32_t *__restrict__ cand_root,
                                                 const uint32_t *__restrict__ count,
                                                 const uint32_t *__restrict__ head,
                                                 const uint16_t *__restrict__ run_box,
                                                 const BoxDev *__restrict__ boxes,
                                                 DevScal *sc, uint32_t *__restrict__ okeys,
                                                 uint32_t *__restrict__ ovals) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const uint32_t nc = sc->nc;
  const int lane = threadIdx.x & 31;
  for (int64_t c0 = gtid() - lane; c0 < (int64_t)nc; c0 += gstride()) {
    const int64_t c = c0 + lane;
    bool ok = false;
    uint32_t root = 0;
    if (c < (int64_t)nc) {
      root = cand_root[c];
      const Geom &g = boxes[run_box[root]].g;
      const double n = (double)count[root];
      ok = true;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const double com = __ddiv_rn(sums[(uint64_t)c * NS + a], n);
        ok &= (com >= g.lo[a]) && (com < g.hi[a]);
      }
    }
    const uint32_t o = warp_slot(ok, &sc->nh);
    if (ok) {
      okeys[o] = head[root];
      ovals[o] = (uint32_t)c;
    }
  }
}

// Halo records (Output_Halos, FOF.c:836-872): means by the reciprocal of n,
// second-moment combinations as written there, all in double, then float.
// The head is reported as an index into the box's own processing order.
template <int NS>
__global__ void __launch_bounds__(kT) k_catalog(const uint32_t *__restrict__ okeys,
                                                const uint32_t *__restrict__ ovals,
                                                const DevScal *__restrict__ sc,
                                                const double *__restrict__ sums,
                                                const uint32_t *__restrict__ cand_root,
                                                const uint32_t *__restrict__ count,
                                                const uint32_t *__restrict__ warn,
                                                const uint16_t *__restrict__ run_box,
                                                uint32_t *__restrict__ boxd, int nbox, int props,
                                                int hs, float *__restrict__ out_props,
                                                uint32_t *__restrict__ head_out,
                                                uint32_t *__restrict__ cat_of_cand,
                                                unsigned long long *n_warn) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const uint32_t nh = sc->nh;
  for (int64_t h = gtid(); h < nh; h += gstride()) {
    const uint32_t c = ovals[h];
    const uint32_t root = cand_root[c];
    const uint32_t n = count[root];
    const int b = run_box[root];
    const double *s = sums + (uint64_t)c * NS;
    const double inv = __ddiv_rn(1.0, (double)n);
    float *rec = out_props + (uint64_t)h * hs;
    int o = 0;
    rec[o++] = (float)n;
    for (int q = 0; q < 6; q++) rec[o++] = __double2float_rn(__dmul_rn(s[q], inv));
    int m = 6;
    if (props & 1) {
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
    if (props & 2) {
      const double VX = s[3], VY = s[4], VZ = s[5];
      const double A[6] = {s[m], s[m + 1], s[m + 2], s[m + 3], s[m + 4], s[m + 5]};
      const double P[6] = {__dmul_rn(VX, VX), __dmul_rn(VY, VY), __dmul_rn(VZ, VZ),
                           __dmul_rn(VX, VY), __dmul_rn(VX, VZ), __dmul_rn(VY, VZ)};
      for (int q = 0; q < 6; q++)
        rec[o++] = __double2float_rn(__dmul_rn(__dsub_rn(A[q], __dmul_rn(P[q], inv)), inv));
    }
    head_out[h] = okeys[h] - boxd[4 * nbox + b];
    cat_of_cand[c] = (uint32_t)h;
    atomicAdd(&boxd[5 * nbox + b], 1u);
    if (warn[c]) atomicAdd(n_warn, 1ull);
  }
}

// First catalog index of each box: owned halos are sorted by processing
// index, which numbers the boxes one after another.
__global__ void k_halo_base(uint32_t *boxd, int nbox) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t acc = 0;
  for (int b = 0; b < nbox; b++) {
    boxd[6 * nbox + b] = acc;
    acc += boxd[5 * nbox + b];
  }
}

// Membership per input particle: the owned halo holding it (or one of its
// images) -- the lowest catalog index when a halo wider than the ghost shell
// leaves two owned copies -- then, in a second pass, the processing index of
// that copy (in its box's numbering) and its stored coordinates.
template <class PT>
__global__ void __launch_bounds__(kT) k_member(const uint32_t *__restrict__ run_of,
                                               const uint32_t *__restrict__ parent,
                                               const uint32_t *__restrict__ cand_of_root,
                                               const uint32_t *__restrict__ cat_of_cand,
                                               const SPos<PT> *__restrict__ spos,
                                               const DevScal *__restrict__ sc,
                                               unsigned long long *__restrict__ member) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const int64_t np = sc->np;
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
    const uint16_t *__restrict__ run_box, const uint32_t *__restrict__ boxd, int nbox,
    const SPos<PT> *__restrict__ spos, const uint32_t *__restrict__ perm,
    const DevScal *__restrict__ sc, const unsigned long long *__restrict__ member,
    uint32_t *__restrict__ member_proc, float *__restrict__ member_pos, Counters *ctr) {
  if (sc->failed) return;  // a sort of this run gave up: its order is not valid
  const int64_t np = sc->np;
  for (int64_t i = gtid(); i < np; i += gstride()) {
    const uint32_t run = run_of[i];
    const uint32_t ci = cand_of_root[parent[run]];
    if (ci == kNone) continue;
    const uint32_t h = cat_of_cand[ci];
    if (h == kNone) continue;
    const SPos<PT> p = spos[i];
    if (member[p.src] == (unsigned long long)h) {
      member_proc[p.src] = perm[i] - boxd[4 * nbox + run_box[run]];
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
// Host side.
// ---------------------------------------------------------------------------

Geom Plan::make_geometry(const cmh_fof_params &p, const std::vector<double> &ltab,
                         int64_t n_in, int cell_factor) const {
  Geom g{};
  double minlink = p.linklength, maxlink = p.linklength;
  if (p.varlink) {
    minlink = maxlink = ltab.empty() ? p.linklength : ltab[0];
    for (double v : ltab) {
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
  if (p.varlink) {
    // the fixed grid of the l(r) rule (FOF.c:50-52, 63-65)
    g.varlink = 1;
    for (int a = 0; a < 3; a++) {
      if (p.ref_cells[a] < 1) fail(CMH_ERR_INVALID_ARGUMENT, "ref_cells must be positive");
      g.origin[a] = p.origin[a];
      g.ref_lcell[a] = (p.hi[a] - p.lo[a] + 2.0 * p.boundary) / p.ref_cells[a];
      g.ref_nc[a] = (int)std::ceil((g.rmax[a] - g.rmin[a]) / g.ref_lcell[a]) + 1;
      if (g.ref_nc[a] >= (1 << 21)) fail(CMH_ERR_CAPACITY, "more than 2^21 grid cells along an axis");
      // the reference scans only neighbouring cells: a longer link would be missed
      if (maxlink > g.ref_lcell[a])
        fail(CMH_ERR_INVALID_ARGUMENT, "linking length longer than the grid cell (raise Px/Py/Pz cells)");
    }
    if (ltab.size() < 2 || !(p.ltab_rmax > 0))
      fail(CMH_ERR_INVALID_ARGUMENT, "variable linking length needs a table of 2+ values");
    g.ltab_n = (int)ltab.size();
    g.ltab_dr = p.ltab_rmax / (double)(g.ltab_n - 1);
  }
  double vol = 1.0;
  for (int a = 0; a < 3; a++) {
    g.G[a] = (int)std::floor((g.rmax[a] - g.rmin[a]) / g.h) + 2;
    if (g.G[a] >= (1 << 21)) fail(CMH_ERR_CAPACITY, "more than 2^21 fine cells along an axis");
    vol *= (g.rmax[a] - g.rmin[a]);
  }
  int k = cell_factor > 0 ? cell_factor : p.cell_factor;
  if (k <= 0) {
    // one top cell per particle on average, as the reference's lcell = L/Px,
    // times the autotuned scale
    const double sep = std::cbrt(vol / std::max<double>((double)n_in, 1.0));
    k = (int)std::lround(sep / g.h * cell_scale);
  }
  if (g.W > kMaxCellFactor)
    fail(CMH_ERR_INVALID_ARGUMENT, "linking lengths span too wide a range (longest / shortest "
                                   "above 18): a fine cell's reach would leave the 27 top cells");
  k = std::min(std::max(k, g.W), kMaxCellFactor);
  while (true) {
    uint64_t T = 1;
    for (int a = 0; a < 3; a++) {
      g.T[a] = (g.G[a] + k - 1) / k;
      T *= (uint64_t)g.T[a];
    }
    if (T < (1ull << 31) || k >= kMaxCellFactor) {
      if (T >= (1ull << 31)) fail(CMH_ERR_CAPACITY, "domain too large for the top-cell grid");
      g.k = k;
      g.k3 = (uint64_t)k * k * k;
      g.kmul = (uint32_t)((1ull << 32) / (uint64_t)k + 1);
      break;
    }
    k++;
  }
  return g;
}

namespace {
// Grid of a grid-stride kernel of kT threads: the CTAs that can be resident
// at once, capped by the work.
template <class K> unsigned rg(K *kernel, int64_t n) {
  return grid_resident(reinterpret_cast<const void *>(kernel), kT, 0, n);
}

// Shared-memory words of one dense top cell: k^3 parents, k^2 bit rows, k^2
// row prefixes and the count of components.
uint64_t dense_words(uint64_t k3all) {
  const uint64_t k = (uint64_t)std::llround(std::cbrt((double)k3all));
  return k3all + 2 * k * k + 1;
}

// Warps per CTA of the dense-top kernel: up to 4, each with the words of one
// top cell, within 200 KiB per CTA.
int dense_warps_per_cta(uint64_t k3all) {
  const uint64_t per = dense_words(k3all) * sizeof(uint32_t);
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(4, (200u << 10) / per));
}

// Occupancy rows of a top cell (k^2).
uint64_t rows_per_top(uint64_t k3all) {
  const uint64_t k = (uint64_t)std::llround(std::cbrt((double)k3all));
  return k * k;
}

// Dense top cells whose rows and row prefixes fit in 4 bytes per processed
// particle plus 1 GiB.
int64_t rows_cap_for(int64_t np_cap, uint64_t k3all) {
  return (int64_t)(((uint64_t)np_cap * 4 + (1ull << 30)) / (rows_per_top(k3all) * 8));
}

bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CMH_CUDA(cudaStreamIsCapturing(s, &cs));
  return cs == cudaStreamCaptureStatusActive;
}

// An event record that other streams can wait on also when it is replayed
// from a recorded graph.
void record_external(cudaEvent_t e, cudaStream_t s) {
  if (capturing(s)) CMH_CUDA(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal));
  else CMH_CUDA(cudaEventRecord(e, s));
}

// Images per input particle expected for a periodic box (the shell's share
// of the padded volume), with headroom for clustering.
double image_estimate(const Geom &g, int64_t n) {
  if (!g.periodic) return 0.0;
  double f = 1.0;
  for (int a = 0; a < 3; a++) f *= (g.L[a] + 2 * g.boundary) / g.L[a];
  return (double)n * (f - 1.0) * 1.5 + 4096.0;
}
}  // namespace

template <class PT>
void Plan::issue(bool want_member, cudaStream_t s, bool timed) {
  const int nbox = (int)boxes_host.size();
  const int64_t n = n_total, npc = np_cap, ncc = nc_cap;
  DevScal *sc = scal.as<DevScal>();
  Counters *c = ctr.as<Counters>();
  unsigned long long *extra = reinterpret_cast<unsigned long long *>(c + 1);  // ngroups, nwarn
  uint32_t *boxd = b_boxd.as<uint32_t>();
  const BoxDev *boxes = b_boxes.as<BoxDev>();
  // buffers whose lifetimes do not overlap share memory: the ingest flags and
  // scans live in arrays of the group stage, and the fine-cell tables run_g
  // and run_of in the unsorted positions, which are dead after the gather
  uint32_t *keep = b_count.as<uint32_t>(), *nimg = b_head.as<uint32_t>();
  uint32_t *keep_scan = b_rtmp1.as<uint32_t>(), *img_scan = b_rtmp2.as<uint32_t>();
  uint64_t *run_g = b_ppos.as<uint64_t>();
  uint32_t *run_of = reinterpret_cast<uint32_t *>(run_g + npc);
  auto mark = [&](int q) {
    if (timed) CMH_CUDA(cudaEventRecord(q < 0 ? ev0 : (q >= 7 ? ev1 : stage_ev[q]), s));
  };
  mark(-1);
  CMH_CUDA(cudaMemsetAsync(scal.p, 0, sizeof(DevScal), s));
  CMH_CUDA(cudaMemsetAsync(ctr.p, 0, sizeof(Counters) + 2 * sizeof(unsigned long long), s));
  CMH_CUDA(cudaMemsetAsync(b_boxd.p, 0, 7 * sizeof(uint32_t) * nbox, s));

  // ---- ingest ----
  // keys and indices are emitted where an odd number of sort passes starts,
  // so that the last pass leaves the indices in b_vals
  const bool odd = radix_order_passes(key_bits) % 2 == 1;
  uint64_t *emit_k = odd ? b_keys_alt.as<uint64_t>() : b_keys.as<uint64_t>();
  uint32_t *emit_v = odd ? b_vals_alt.as<uint32_t>() : b_vals.as<uint32_t>();
  if (n > 0) {
    k_ingest_count<PT><<<rg(k_ingest_count<PT>, n), kT, 0, s>>>(boxes, nbox, n, keep,
                                                      nimg);
    CMH_LAUNCHED();
  }
  // the keep and image scans side by side (the image scan on the second
  // stream, with its own scratch)
  CMH_CUDA(cudaEventRecord(ev_fork, s));
  CMH_CUDA(cudaStreamWaitEvent(bf_stream, ev_fork, 0));
  exclusive_scan_u32(nimg, img_scan, n, &sc->img_total, scan_tmp2, bf_stream);
  CMH_CUDA(cudaEventRecord(ev_join, bf_stream));
  // then, on that stream, the clearing of the later stages' tables, which
  // overlaps the ingest and the sort (their first users wait for it)
  const int NS = 6 + ((props & 1) ? 6 : 0) + ((props & 2) ? 6 : 0);
  CMH_CUDA(cudaMemsetAsync(b_top_range.p, 0, n_top * 8, bf_stream));
  CMH_CUDA(cudaMemsetAsync(b_top_slot.p, 0xff, n_top * 4, bf_stream));
  CMH_CUDA(cudaMemsetAsync(b_cand_of_root.p, 0xff, npc * 4, bf_stream));
  CMH_CUDA(cudaMemsetAsync(b_sums.p, 0, (size_t)ncc * NS * 8, bf_stream));
  CMH_CUDA(cudaMemsetAsync(b_warn.p, 0, (size_t)ncc * 4, bf_stream));
  CMH_CUDA(cudaMemsetAsync(b_cat_of_cand.p, 0xff, (size_t)ncc * 4, bf_stream));
  if (want_member && n > 0) {
    CMH_CUDA(cudaMemsetAsync(b_member.p, 0xff, (size_t)n * 8, bf_stream));
    CMH_CUDA(cudaMemsetAsync(b_member_proc.p, 0xff, (size_t)n * 4, bf_stream));
    CMH_CUDA(cudaMemsetAsync(b_member_pos.p, 0, (size_t)n * 12, bf_stream));
  }
  CMH_CUDA(cudaEventRecord(ev_cleared, bf_stream));
  exclusive_scan_u32(keep, keep_scan, n, &sc->kept_total, scan_tmp, s);
  CMH_CUDA(cudaStreamWaitEvent(s, ev_join, 0));
  k_box_totals<<<1, 32, 0, s>>>(boxes, nbox, n, keep_scan,
                                img_scan, sc, boxd, (uint32_t)npc);
  CMH_LAUNCHED();
  if (n > 0) {
    k_ingest_emit<PT><<<rg(k_ingest_emit<PT>, n), kT, 0, s>>>(
        boxes, nbox, n, k3all, keep, keep_scan,
        img_scan, nimg, boxd, (uint32_t)npc,
        emit_k, emit_v, b_ppos.as<SPos<PT>>());
    CMH_LAUNCHED();
  }
  mark(0);
  // the ingest's flag arrays become the group counts and heads: cleared on
  // the second stream once the emission has read them
  CMH_CUDA(cudaEventRecord(ev_emitted, s));
  CMH_CUDA(cudaStreamWaitEvent(bf_stream, ev_emitted, 0));
  CMH_CUDA(cudaMemsetAsync(b_count.p, 0, npc * 4, bf_stream));
  CMH_CUDA(cudaMemsetAsync(b_head.p, 0xff, npc * 4, bf_stream));
  CMH_CUDA(cudaEventRecord(ev_cleared2, bf_stream));
  // host inputs: their positions are read no more (a next run's may be
  // copied into their buffer)
  if (vel_wait) record_external(ev_pos_free, s);
  // ---- sort ----
  // the sort leaves the indices in cell order in b_vals and no sorted keys:
  // k_gather_flags recomputes the fine cells into b_keys from the positions
  // a look-back that gives up raises sc->failed, and every later kernel of
  // the run then returns at once (the order would not be valid)
  radix_order_u64_u32(emit_k, emit_v, odd ? b_keys.as<uint64_t>() : b_keys_alt.as<uint64_t>(),
                      odd ? b_vals.as<uint32_t>() : b_vals_alt.as<uint32_t>(), npc, &sc->np,
                      key_bits, sort_tmp, &sc->failed, s,
                      SortWaits{spin_cap, stall_sort ? 1u : 0xffffffffu});
  mark(1);
  // ---- runs, top-cell ranges, dense top cells ----
  uint32_t *flag = b_keys_alt.as<uint32_t>();  // reuse: [flag | run_scan]
  uint32_t *run_scan = flag + npc;
  k_gather_flags<PT><<<rg(k_gather_flags<PT>, npc), kT, 0, s>>>(
      b_vals.as<uint32_t>(), b_ppos.as<SPos<PT>>(), boxes, nbox, b_spos.as<SPos<PT>>(),
      b_keys.as<uint64_t>(), flag, sc);
  CMH_LAUNCHED();
  exclusive_scan_u32(flag, run_scan, npc, &sc->R, scan_tmp, s, &sc->np);
  CMH_CUDA(cudaStreamWaitEvent(s, ev_cleared, 0));  // top ranges and slots cleared
  k_runs<PT><<<rg(k_runs<PT>, npc), kT, 0, s>>>(b_keys.as<uint64_t>(), flag, run_scan,
                                               b_spos.as<SPos<PT>>(), boxes, nbox, sc, run_of,
                                               b_run_start.as<uint32_t>(), run_g,
                                               b_run_box.as<uint16_t>(), b_parent.as<uint32_t>(),
                                               b_top_range.as<uint32_t>());
  CMH_LAUNCHED();
  if (varlink) {
    if (fp32)
      k_varlink_recs<PT, true><<<rg(k_varlink_recs<PT, true>, npc), kT, 0, s>>>(b_spos.as<SPos<PT>>(), run_of,
                                                 b_run_box.as<uint16_t>(), boxes, sc,
                                                 b_svl.as<VLRec64>());
    else
      k_varlink_recs<PT, false><<<rg(k_varlink_recs<PT, false>, npc), kT, 0, s>>>(b_spos.as<SPos<PT>>(), run_of,
                                                  b_run_box.as<uint16_t>(), boxes, sc,
                                                  b_svl.as<VLRec64>());
    CMH_LAUNCHED();
  }
  k_dense_pick<<<rg(k_dense_pick, npc), kT, 0, s>>>(
      run_g, b_run_box.as<uint16_t>(), boxes, sc, b_top_range.as<uint2>(), dense_min,
      (uint32_t)nd_cap, b_top_slot.as<uint32_t>(), b_dense_range.as<uint2>(),
      b_dense_big.as<uint32_t>());
  CMH_LAUNCHED();
  mark(2);
  // ---- befriending: dense top cells inside (CTA each) on a second stream
  // while the sparse fast path runs (both join cells through the lock-free
  // union-find), then the queued cells' warp path, near then far ----
  uint32_t *queue = b_rtmp1.as<uint32_t>();  // the keep scan's, free since the emission
  const int dwpc = dense_warps_per_cta(k3all);
  const uint32_t kk = (uint32_t)rows_per_top(k3all);
  const size_t dsm = (size_t)dwpc * dense_words(k3all) * sizeof(uint32_t);
  const unsigned gd = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>((nd_cap + dwpc - 1) / dwpc, (int64_t)kSMs * 64 / dwpc));
  auto befriend = [&](auto fp32_tag, auto vl_tag) {
    constexpr bool FP = decltype(fp32_tag)::value;
    constexpr bool VL = decltype(vl_tag)::value;
    const VLRec<FP> *svl = VL ? b_svl.as<VLRec<FP>>() : nullptr;
    // dense top cells on a second stream, beside the sparse cells
    CMH_CUDA(cudaEventRecord(ev_fork, s));
    CMH_CUDA(cudaStreamWaitEvent(bf_stream, ev_fork, 0));
    k_befriend_dense<PT, FP, VL><<<gd, 32 * dwpc, dsm, bf_stream>>>(
        boxes, b_run_box.as<uint16_t>(), k3all, b_run_start.as<uint32_t>(),
        run_g, b_dense_range.as<uint2>(), b_dense_big.as<uint32_t>(), sc, (uint32_t)nd_cap,
        b_rows.as<uint32_t>(), kk, b_spos.as<SPos<PT>>(), svl, b_parent.as<uint32_t>(), c,
        (uint32_t)dense_words(k3all));
    CMH_LAUNCHED();
    CMH_CUDA(cudaEventRecord(ev_join, bf_stream));
    k_befriend_simple<PT, FP, VL><<<rg(k_befriend_simple<PT, FP, VL>, npc), kT, 0, s>>>(
        boxes, b_run_box.as<uint16_t>(), b_run_start.as<uint32_t>(), run_g,
        sc, b_top_range.as<uint2>(), b_top_slot.as<uint32_t>(),
        b_spos.as<SPos<PT>>(), svl, b_parent.as<uint32_t>(), queue, c);
    CMH_LAUNCHED();
    CMH_CUDA(cudaStreamWaitEvent(s, ev_join, 0));
    k_befriend<PT, FP, VL, 0><<<rg(k_befriend<PT, FP, VL, 0>, npc * 32), kT, 0, s>>>(
        boxes, b_run_box.as<uint16_t>(), k3all, b_run_start.as<uint32_t>(),
        run_g, queue, sc, b_top_range.as<uint2>(), b_top_slot.as<uint32_t>(),
        b_rows.as<uint32_t>(), kk, b_spos.as<SPos<PT>>(), svl, b_parent.as<uint32_t>(), c);
    CMH_LAUNCHED();
    k_compress<<<rg(k_compress, npc), kT, 0, s>>>(b_parent.as<uint32_t>(), sc);
    CMH_LAUNCHED();
    k_befriend<PT, FP, VL, 1><<<rg(k_befriend<PT, FP, VL, 1>, npc * 32), kT, 0, s>>>(
        boxes, b_run_box.as<uint16_t>(), k3all, b_run_start.as<uint32_t>(),
        run_g, queue, sc, b_top_range.as<uint2>(), b_top_slot.as<uint32_t>(),
        b_rows.as<uint32_t>(), kk, b_spos.as<SPos<PT>>(), svl, b_parent.as<uint32_t>(), c);
    CMH_LAUNCHED();
  };
  if (fp32 && varlink) befriend(std::true_type{}, std::true_type{});
  else if (fp32) befriend(std::true_type{}, std::false_type{});
  else if (varlink) befriend(std::false_type{}, std::true_type{});
  else befriend(std::false_type{}, std::false_type{});
  k_compress<<<rg(k_compress, npc), kT, 0, s>>>(b_parent.as<uint32_t>(), sc);
  CMH_LAUNCHED();
  mark(3);

  // ---- groups, candidates ----
  CMH_CUDA(cudaStreamWaitEvent(s, ev_cleared2, 0));  // counts and heads cleared
  k_group_count<<<rg(k_group_count, npc), kT, 0, s>>>(run_of, b_parent.as<uint32_t>(),
                                  b_vals.as<uint32_t>(), sc, b_count.as<uint32_t>(),
                                  b_head.as<uint32_t>());
  CMH_LAUNCHED();
  if (sampling && n > 0) {
    CMH_CUDA(cudaMemsetAsync(b_samp.p, 0, (size_t)n, s));
    k_subsample<PT><<<rg(k_subsample<PT>, npc), kT, 0, s>>>(
        run_of, b_parent.as<uint32_t>(), b_count.as<uint32_t>(), b_vals.as<uint32_t>(),
        b_spos.as<SPos<PT>>(), b_run_box.as<uint16_t>(), boxes, boxd, nbox, sc, samp_ids,
        samp_in, samp_out, samp_seed, samp_closed, b_samp.as<uint8_t>());
    CMH_LAUNCHED();
  }
  k_cand_pick<<<rg(k_cand_pick, npc), kT, 0, s>>>(
      b_parent.as<uint32_t>(), b_count.as<uint32_t>(), b_run_box.as<uint16_t>(), boxes, sc,
      b_cand_of_root.as<uint32_t>(), b_cand_root.as<uint32_t>(), extra + 0);
  CMH_LAUNCHED();
  mark(4);

  // ---- property sums, ownership, catalog ----
  if (vel_wait) {
    // host-resident velocities arrive on the side stream while the steps
    // above run; the sums are their first reader
    CMH_CUDA(cudaStreamWaitEvent(s, ev_vel_ready,
                                 capturing(s) ? cudaEventWaitExternal : cudaEventWaitDefault));
  }
#define CMH_SUMS(NSV)                                                                         \
  k_group_sums<PT, NSV><<<rg(k_group_sums<PT, NSV>, npc), kT, 0, s>>>(run_of, b_parent.as<uint32_t>(),  \
                                          b_cand_of_root.as<uint32_t>(),                      \
                                          b_run_box.as<uint16_t>(), boxes,                    \
                                          b_spos.as<SPos<PT>>(), sc, props,                   \
                                          b_sums.as<double>(), b_warn.as<uint32_t>())
  if (NS == 6) CMH_SUMS(6);
  else if (NS == 12) CMH_SUMS(12);
  else CMH_SUMS(18);
#undef CMH_SUMS
  CMH_LAUNCHED();
  mark(5);
  if (vel_wait) record_external(ev_vel_free, s);  // nor their velocities
#define CMH_OWNED(NSV)                                                                          \
  k_own_pick<NSV><<<rg(k_own_pick<NSV>, ncc), kT, 0, s>>>(                                      \
      b_sums.as<double>(), b_cand_root.as<uint32_t>(), b_count.as<uint32_t>(),                  \
      b_head.as<uint32_t>(), b_run_box.as<uint16_t>(), boxes, sc, b_okeys.as<uint32_t>(),       \
      b_ovals.as<uint32_t>())
  if (NS == 6) CMH_OWNED(6);
  else if (NS == 12) CMH_OWNED(12);
  else CMH_OWNED(18);
#undef CMH_OWNED
  CMH_LAUNCHED();
  radix_sort_u32_u32(b_okeys.as<uint32_t>(), b_ovals.as<uint32_t>(), b_okeys_alt.as<uint32_t>(),
                     b_ovals_alt.as<uint32_t>(), ncc, &sc->nh, bits_for((uint64_t)npc),
                     sort_tmp, &sc->failed, s, SortWaits{spin_cap, 0xffffffffu});
#define CMH_CATALOG(NSV)                                                                        \
  k_catalog<NSV><<<rg(k_catalog<NSV>, ncc), kT, 0, s>>>(b_okeys.as<uint32_t>(), b_ovals.as<uint32_t>(), sc,          \
                                   b_sums.as<double>(), b_cand_root.as<uint32_t>(),             \
                                   b_count.as<uint32_t>(), b_warn.as<uint32_t>(),               \
                                   b_run_box.as<uint16_t>(), boxd, nbox, props, hs,              \
                                   b_props.as<float>(), b_head_out.as<uint32_t>(),              \
                                   b_cat_of_cand.as<uint32_t>(), extra + 1)
  if (NS == 6) CMH_CATALOG(6);
  else if (NS == 12) CMH_CATALOG(12);
  else CMH_CATALOG(18);
#undef CMH_CATALOG
  CMH_LAUNCHED();
  k_halo_base<<<1, 32, 0, s>>>(boxd, nbox);
  CMH_LAUNCHED();
  mark(6);
  if (want_member && n > 0) {
    k_member<PT><<<rg(k_member<PT>, npc), kT, 0, s>>>(run_of, b_parent.as<uint32_t>(),
                                   b_cand_of_root.as<uint32_t>(), b_cat_of_cand.as<uint32_t>(),
                                   b_spos.as<SPos<PT>>(), sc, b_member.as<unsigned long long>());
    CMH_LAUNCHED();
    k_member_copy<PT><<<rg(k_member_copy<PT>, npc), kT, 0, s>>>(
        run_of, b_parent.as<uint32_t>(), b_cand_of_root.as<uint32_t>(),
        b_cat_of_cand.as<uint32_t>(), b_run_box.as<uint16_t>(), boxd, nbox,
        b_spos.as<SPos<PT>>(), b_vals.as<uint32_t>(), sc, b_member.as<unsigned long long>(),
        b_member_proc.as<uint32_t>(), b_member_pos.as<float>(), c);
    CMH_LAUNCHED();
  }
  mark(7);
}

void Plan::prepare(const std::vector<BoxSpec> &specs, bool want_member) {
  if (!bf_stream) {
    CMH_CUDA(cudaStreamCreateWithFlags(&bf_stream, cudaStreamNonBlocking));
    CMH_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    CMH_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    CMH_CUDA(cudaEventCreateWithFlags(&ev_cleared, cudaEventDisableTiming));
    CMH_CUDA(cudaEventCreateWithFlags(&ev_emitted, cudaEventDisableTiming));
    CMH_CUDA(cudaEventCreateWithFlags(&ev_cleared2, cudaEventDisableTiming));
  }
  const int nbox = (int)specs.size();
  if (nbox < 1 || nbox > kMaxBoxes) fail(CMH_ERR_INVALID_ARGUMENT, "1 to 1024 boxes per run");
  boxes_host.resize(nbox);
  n_total = 0;
  uint64_t tops = 0;
  int kmax = 1;
  double img = 0.0;
  props = -1;
  for (int b = 0; b < nbox; b++) {
    const BoxSpec &sp = specs[b];
    BoxDev &bd = boxes_host[b];
    memset(&bd, 0, sizeof bd);
    bd.g = make_geometry(sp.params, sp.ltab, sp.n, sp.cell_factor);
    bd.g.union_cap = union_cap;
    if (props < 0) props = bd.g.props;
    if (bd.g.props != props) fail(CMH_ERR_INVALID_ARGUMENT, "boxes of a run share the property set");
    bd.pos = sp.pos;
    bd.vel = sp.vel;
    bd.vel_f64 = sp.vel_f64 ? 1 : 0;
    bd.n = (uint32_t)sp.n;
    bd.in_base = (uint64_t)n_total;
    bd.top_base = tops;
    n_total += sp.n;
    tops += (uint64_t)bd.g.T[0] * bd.g.T[1] * bd.g.T[2];
    kmax = std::max(kmax, bd.g.k);
    img += image_estimate(bd.g, sp.n);
  }
  if (n_total >= (int64_t)0xfffffff0ll) fail(CMH_ERR_CAPACITY, "more than 2^32 input particles in a run");
  // linking-length tables of all boxes, one device array
  varlink = false;
  ltab_all.clear();
  for (int b = 0; b < nbox; b++)
    if (boxes_host[b].g.varlink) {
      varlink = true;
      ltab_all.insert(ltab_all.end(), specs[b].ltab.begin(), specs[b].ltab.end());
    }
  if (varlink) {
    ltab_dev.ensure(ltab_all.size() * sizeof(double));
    size_t off = 0;
    for (int b = 0; b < nbox; b++)
      if (boxes_host[b].g.varlink) {
        boxes_host[b].g.ltab = ltab_dev.as<double>() + off;
        off += specs[b].ltab.size();
      }
  }
  hs = 7 + ((props & 1) ? 6 : 0) + ((props & 2) ? 6 : 0);
  k3all = (uint64_t)kmax * kmax * kmax;
  n_top = tops;
  key_bits = bits_for(tops * k3all - 1);
  if (tops >= (1ull << 40) || key_bits > 62) fail(CMH_ERR_CAPACITY, "too many cells in a run");
  // capacities: grown after a run that overflowed them, never shrunk
  const int64_t want_np = std::min<int64_t>(n_total + (int64_t)img, (int64_t)0xfffffff0ll);
  np_cap = std::max<int64_t>(np_cap, std::max<int64_t>(want_np, 1));
  // dense top cells: their rows take at most 4 bytes per processed particle
  // plus 1 GiB (dense top cells past the cap are scanned instead)
  nd_cap = std::max<int64_t>(nd_cap, np_cap / 1024 + 1024);
  nd_cap = std::min<int64_t>(nd_cap, std::max<int64_t>(1024, rows_cap_for(np_cap, k3all)));
  double mincut = 1e300;
  for (const BoxDev &bd : boxes_host) mincut = std::min(mincut, bd.g.nphalomin);
  const int64_t div = (int64_t)std::max(1.0, std::floor(mincut));
  nc_cap = std::max<int64_t>(1, np_cap / div + 1);

  const int64_t nn = std::max<int64_t>(n_total, 1), npc = np_cap, ncc = nc_cap;
  scal.ensure(sizeof(DevScal));
  ctr.ensure(sizeof(Counters) + 2 * sizeof(unsigned long long));
  b_boxes.ensure(sizeof(BoxDev) * nbox);
  b_boxd.ensure(sizeof(uint32_t) * 7 * nbox);
  b_keys.ensure(npc * 8);
  b_keys_alt.ensure(npc * 8);
  b_vals.ensure(npc * 4);
  b_vals_alt.ensure(npc * 4);
  const size_t rec = pos_dtype == CMH_FLOAT64 ? sizeof(SPos<double>) : sizeof(SPos<float>);
  b_ppos.ensure(npc * rec);
  b_spos.ensure(npc * rec);
  if (varlink) b_svl.ensure(npc * sizeof(VLRec64));
  b_run_start.ensure((npc + 1) * 4);
  b_run_box.ensure(npc * 2);
  b_top_range.ensure(n_top * 8);
  b_top_slot.ensure(n_top * 4);
  b_rtmp1.ensure(npc * 4);
  b_rtmp2.ensure(npc * 4);
  b_rows.ensure((size_t)nd_cap * rows_per_top(k3all) * 2 * sizeof(uint32_t));
  b_dense_range.ensure((size_t)nd_cap * sizeof(uint2));
  b_dense_big.ensure((size_t)nd_cap * sizeof(uint32_t));
  b_parent.ensure(npc * 4);
  b_count.ensure(npc * 4);
  b_head.ensure(npc * 4);
  b_cand_of_root.ensure(npc * 4);
  if (sampling) b_samp.ensure((size_t)nn);
  b_cand_root.ensure(ncc * 4);
  b_sums.ensure(ncc * 18 * 8);
  b_warn.ensure(ncc * 4);
  b_okeys.ensure(ncc * 4);
  b_ovals.ensure(ncc * 4);
  b_okeys_alt.ensure(ncc * 4);
  b_ovals_alt.ensure(ncc * 4);
  b_props.ensure(ncc * hs * 4);
  b_head_out.ensure(ncc * 4);
  b_cat_of_cand.ensure(ncc * 4);
  if (want_member) {
    b_member.ensure(nn * 8);
    b_member_proc.ensure(nn * 4);
    b_member_pos.ensure(nn * 12);
  }
  // shared memory of the dense-top kernel: one parent per fine cell of a top
  // cell (set here, outside any graph capture)
  {
    const int dsm = (int)(dense_warps_per_cta(k3all) * dense_words(k3all) * sizeof(uint32_t));
    const void *dense[] = {
        (const void *)k_befriend_dense<float, true, false>,
        (const void *)k_befriend_dense<float, false, false>,
        (const void *)k_befriend_dense<double, true, false>,
        (const void *)k_befriend_dense<double, false, false>,
        (const void *)k_befriend_dense<float, true, true>,
        (const void *)k_befriend_dense<float, false, true>,
        (const void *)k_befriend_dense<double, true, true>,
        (const void *)k_befriend_dense<double, false, true>};
    for (const void *f : dense)
      CMH_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, dsm));
  }
  // pre-grow the scratch of the scans and sorts so that issue() allocates
  // nothing (it may be captured in a graph)
  {
    int64_t need = 0;
    for (int64_t m = std::max(npc, nn) * 1; m > 4096;) {
      m = (m + 4095) / 4096;
      need += 2 * m;
    }
    scan_tmp.ensure((size_t)(need + 16) * sizeof(uint32_t));
    scan_tmp2.ensure((size_t)(need + 16) * sizeof(uint32_t));
    sort_tmp.ensure(radix_sort_scratch(std::max(npc, ncc)));
  }
}

void Plan::read_back(cudaStream_t s, bool timed) {
  const int nbox = (int)boxes_host.size();
  struct {
    Counters c;
    unsigned long long ngroups, nwarn;
  } hc;
  DevScal hs_;
  CMH_CUDA(cudaMemcpyAsync(&hc, ctr.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
  CMH_CUDA(cudaMemcpyAsync(&hs_, scal.p, sizeof(DevScal), cudaMemcpyDeviceToHost, s));
  boxd_host.resize(7 * nbox);
  CMH_CUDA(cudaMemcpyAsync(boxd_host.data(), b_boxd.p, sizeof(uint32_t) * 7 * nbox,
                           cudaMemcpyDeviceToHost, s));
  CMH_CUDA(cudaStreamSynchronize(s));
  last = hs_;
  // CMH_FAULT=overflow: the run is treated as having outgrown its buffers, so
  // it is repeated with room until the attempts run out (CMH_ERR_CAPACITY),
  // as a rank whose receive buffer overflows stops (read_data.c:551-556)
  if (fault_active("overflow")) last.overflow |= 1u;
  if (hc.c.uf_giveups)
    fail(CMH_ERR_DEVICE_TIMEOUT, "union-find retry loop reached its iteration cap");
  if (hs_.failed)
    fail(CMH_ERR_DEVICE_TIMEOUT, "radix sort look-back wait reached its cap");
  stats = cmh_stats{};
  stats.n_in = n_total;
  stats.n_out = n_total - hs_.kept_total;
  stats.n_images = hs_.img_total;
  stats.n_proc = hs_.np;
  stats.n_cells = hs_.R;
  stats.n_groups = (int64_t)hc.ngroups;
  stats.n_candidates = hs_.nc;
  stats.nhalos = hs_.nh;
  stats.n_edge_warn = (int64_t)hc.nwarn;
  stats.n_pair_tests = (int64_t)hc.c.pair_tests;
  stats.n_rechecks = (int64_t)hc.c.rechecks;
  stats.n_member_conflicts = (int64_t)hc.c.member_conflicts;
  stats.cell_factor = boxes_host[0].g.k;
  stats.key_bits = key_bits;
  stats.n_cell_pairs = (int64_t)hc.c.cand_pairs;
  stats.n_root_skips = (int64_t)hc.c.root_skips;
  stats.n_unions = (int64_t)hc.c.unions;
  stats.n_find_steps = (int64_t)hc.c.find_steps;
  stats.n_scan_iters = (int64_t)hc.c.scan_iters;
  stats.n_window_iters = (int64_t)hc.c.window_iters;
  stats.n_dense_tops = hs_.nd;
  stats.n_queued = hs_.qcount;
  stats.n_big_tops = hs_.nbig;
  if (timed) {
    float ms = 0;
    CMH_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    stats.ms_total = ms;
    cudaEvent_t b[9] = {ev0, stage_ev[0], stage_ev[1], stage_ev[2], stage_ev[3],
                        stage_ev[4], stage_ev[5], stage_ev[6], ev1};
    for (int q = 0; q < 8; q++) CMH_CUDA(cudaEventElapsedTime(&stats.stage_ms[q], b[q], b[q + 1]));
  }
  out_nhalos = hs_.nh;
}

void Plan::run_batch(const std::vector<BoxSpec> &specs, bool want_member, cudaStream_t s) {
  CMH_CUDA(cudaSetDevice(device));
  overwritten = false;
  for (int attempt = 0; attempt < 3; attempt++) {
    prepare(specs, want_member);
    // the graph stays valid while the inputs, sizes and capacities do
    std::vector<unsigned char> sig(sizeof(BoxDev) * boxes_host.size());
    memcpy(sig.data(), boxes_host.data(), sig.size());
    int64_t samp_bits[3] = {0, 0, 0};
    memcpy(&samp_bits[0], &samp_in, 8);
    memcpy(&samp_bits[1], &samp_out, 8);
    samp_bits[2] = (int64_t)samp_seed ^ ((int64_t)samp_closed << 40);
    stall_sort = fault_active("lookback");
    const int64_t caps[12] = {np_cap, nd_cap, nc_cap, (int64_t)want_member, (int64_t)fp32,
                              (int64_t)dense_min, (int64_t)vel_wait,
                              sampling ? samp_bits[0] : -1, samp_bits[1],
                              samp_bits[2] ^ (int64_t)(uintptr_t)samp_ids,
                              (int64_t)spin_cap, (int64_t)stall_sort};
    sig.insert(sig.end(), (const unsigned char *)caps, (const unsigned char *)caps + sizeof caps);
    // and the workspace addresses the recorded launches use
    each_buf([&](DevBuf &b) {
      sig.insert(sig.end(), (const unsigned char *)&b.p, (const unsigned char *)&b.p + sizeof b.p);
    });
    sig.insert(sig.end(), (const unsigned char *)ltab_all.data(),
               (const unsigned char *)(ltab_all.data() + ltab_all.size()));
    int slot = -1;  // the recorded graph of this shape, if any
    for (int q = 0; q < 2; q++)
      if (graph_exec[q] && sig == graph_sig[q]) slot = q;
    const bool same = slot >= 0;
    // the device box table (and length tables) hold the last uploaded shape,
    // which an eager run of another shape may have replaced since the graph
    // was recorded: upload whenever they differ from this run's
    if (sig != uploaded_sig) {
      uploaded_sig.clear();
      CMH_CUDA(cudaMemcpyAsync(b_boxes.p, boxes_host.data(), sizeof(BoxDev) * boxes_host.size(),
                               cudaMemcpyHostToDevice, s));
      if (varlink)
        CMH_CUDA(cudaMemcpyAsync(ltab_dev.p, ltab_all.data(), ltab_all.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
      CMH_CUDA(cudaStreamSynchronize(s));
      uploaded_sig = sig;
    }
    const long long l0 = g_launches;
    if (use_graph && same) {
      // a replay is timed as a whole; stage times come from eager runs
      CMH_CUDA(cudaEventRecord(ev0, s));
      CMH_CUDA(cudaGraphLaunch(graph_exec[slot], s));
      graph_next = 1 - slot;  // keep the one just used
      CMH_CUDA(cudaEventRecord(ev1, s));
      launches_per_run_graph_ok = true;
      queue_pending();
      read_back(s, false);
      CMH_CUDA(cudaEventElapsedTime(&stats.ms_total, ev0, ev1));
    } else {
      if (pos_dtype == CMH_FLOAT64) issue<double>(want_member, s, true);
      else issue<float>(want_member, s, true);
      queue_pending();
      read_back(s, true);
      launches_per_run = (int32_t)(g_launches - l0);
      if (!(last.overflow & 1u) && use_graph) capture(want_member, s, sig);
    }
    stats.n_launches = launches_per_run;
    if (last.overflow & 2u)  // faster next time, within the rows budget
      nd_cap = std::min<int64_t>((int64_t)last.nd + last.nd / 4 + 256,
                                 std::max<int64_t>(nd_cap, rows_cap_for(np_cap, k3all)));
    if (!(last.overflow & 1u)) return;
    np_cap = (int64_t)last.np_raw + last.np_raw / 8 + 4096;  // repeat with room
    if (overwritten) {
      // one input buffer, already refilled with the next run's inputs: this
      // run's are copied again, and the next run's wait for the repeat
      CMH_CUDA(cudaStreamSynchronize(side_stream));
      staged.front().pending = true;
      overwritten = false;
      stage_inputs(cur_host.data(), (int)cur_host.size(), s, 0);
      CMH_CUDA(cudaStreamWaitEvent(s, ev_pos[0], 0));
      ev_vel_ready = ev_vel[0];
    }
  }
  fail(CMH_ERR_CAPACITY, "processed particles kept outgrowing the buffers");
}

void Plan::capture(bool want_member, cudaStream_t s, const std::vector<unsigned char> &sig) {
  const int q = graph_next;
  graph_next = 1 - q;
  if (graph_exec[q]) {
    cudaGraphExecDestroy(graph_exec[q]);
    graph_exec[q] = nullptr;
    graph_sig[q].clear();
  }
  // recorded on the plan's own stream (the legacy stream cannot be
  // captured); the graph is then launched on the caller's stream
  if (!cap_stream) CMH_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
  cudaGraph_t graph = nullptr;
  CMH_CUDA(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
  try {
    if (pos_dtype == CMH_FLOAT64) issue<double>(want_member, cap_stream, false);
    else issue<float>(want_member, cap_stream, false);
  } catch (...) {
    cudaStreamEndCapture(cap_stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  CMH_CUDA(cudaStreamEndCapture(cap_stream, &graph));
  cudaError_t e = cudaGraphInstantiate(&graph_exec[q], graph, 0);
  cudaGraphDestroy(graph);
  CMH_CUDA(e);
  graph_sig[q] = sig;
  (void)s;
}

// Grid search over the cell-size scale and the dense-top threshold, timing
// eager runs of the real boxes (after one untimed run per setting, which
// also grows the buffers).  The fastest setting stays in the plan.
cmh_tuning Plan::autotune(const std::vector<BoxSpec> &specs, int repeats, cudaStream_t s) {
  const double scales[] = {0.5, 0.75, 1.0, 1.5, 2.0};
  const uint32_t mins[] = {8, 16, 32};
  const bool graph0 = use_graph;
  use_graph = false;
  cmh_tuning best{cell_scale, (int32_t)dense_min, 1e30f, 0};
  for (double sc : scales)
    for (uint32_t dm : mins) {
      cell_scale = sc;
      dense_min = dm;
      // each setting starts from an empty workspace, so that one setting's
      // large buffers (many top cells, or many dense ones) do not stay allocated
      // under the next; a setting that does not fit in memory is skipped
      release_workspace();
      float t = 0;
      try {
        run_batch(specs, false, s);
        for (int r = 0; r < std::max(repeats, 1); r++) {
          run_batch(specs, false, s);
          t += stats.ms_total;
        }
      } catch (const Error &e) {
        if (e.code != CMH_ERR_OUT_OF_MEMORY) {
          use_graph = graph0;
          throw;
        }
        continue;
      }
      t /= std::max(repeats, 1);
      best.tried++;
      if (t < best.ms) {
        best.ms = t;
        best.cell_scale = sc;
        best.dense_min = (int32_t)dm;
      }
    }
  release_workspace();
  use_graph = graph0;
  if (best.tried == 0) fail(CMH_ERR_OUT_OF_MEMORY, "no setting of the autotuner fits in memory");
  cell_scale = best.cell_scale;
  dense_min = (uint32_t)best.dense_min;
  return best;
}

namespace {
// Byte offsets of each box's positions and velocities in the input buffers
// (256-byte aligned slices); returns the totals.
void input_layout(const cmh_particles *parts, int nbox, std::vector<size_t> *opos,
                  std::vector<size_t> *ovel, size_t *tpos, size_t *tvel) {
  size_t p = 0, v = 0;
  opos->resize(nbox);
  ovel->resize(nbox);
  for (int i = 0; i < nbox; i++) {
    (*opos)[i] = p;
    (*ovel)[i] = v;
    p += ((size_t)parts[i].n * 3 * (parts[i].pos_dtype == CMH_FLOAT64 ? 8 : 4) + 255) & ~(size_t)255;
    v += ((size_t)parts[i].n * 3 * (parts[i].vel_dtype == CMH_FLOAT64 ? 8 : 4) + 255) & ~(size_t)255;
  }
  *tpos = p;
  *tvel = v;
}

bool same_inputs(const std::vector<cmh_particles> &a, const cmh_particles *b, int nbox) {
  if ((int)a.size() != nbox) return false;
  for (int i = 0; i < nbox; i++)
    if (a[i].pos != b[i].pos || a[i].vel != b[i].vel || a[i].n != b[i].n ||
        a[i].pos_dtype != b[i].pos_dtype || a[i].vel_dtype != b[i].vel_dtype)
      return false;
  return true;
}
}  // namespace

void Plan::ensure_side() {
  if (side_stream) return;
  CMH_CUDA(cudaStreamCreateWithFlags(&side_stream, cudaStreamNonBlocking));
  CMH_CUDA(cudaEventCreateWithFlags(&ev_side_start, cudaEventDisableTiming));
  CMH_CUDA(cudaEventCreateWithFlags(&ev_pos_free, cudaEventDisableTiming));
  CMH_CUDA(cudaEventCreateWithFlags(&ev_vel_free, cudaEventDisableTiming));
  for (int b = 0; b < 2; b++) {
    CMH_CUDA(cudaEventCreateWithFlags(&ev_pos[b], cudaEventDisableTiming));
    CMH_CUDA(cudaEventCreateWithFlags(&ev_vel[b], cudaEventDisableTiming));
  }
}

int Plan::stage_inputs(const cmh_particles *parts, int nbox, cudaStream_t s, int b) {
  CMH_CUDA(cudaSetDevice(device));
  ensure_side();
  std::vector<size_t> opos, ovel;
  size_t tpos, tvel;
  input_layout(parts, nbox, &opos, &ovel, &tpos, &tvel);
  in_pos[b].ensure(std::max<size_t>(tpos, 256));
  in_vel[b].ensure(std::max<size_t>(tvel, 256));
  // after the caller's queued work (a run that read this buffer before), on
  // the side stream: the positions first, at the link's full bandwidth
  CMH_CUDA(cudaEventRecord(ev_side_start, s));
  CMH_CUDA(cudaStreamWaitEvent(side_stream, ev_side_start, 0));
  copy_inputs(parts, nbox, b, false);
  return b;
}

// The copies of staged host inputs into buffer b on the side stream, every
// box's positions before any velocities.  `behind_run`: the positions wait
// for the queued run's ingest and the velocities for its property sums.
void Plan::copy_inputs(const cmh_particles *parts, int nbox, int b, bool behind_run) {
  std::vector<size_t> opos, ovel;
  size_t tpos, tvel;
  input_layout(parts, nbox, &opos, &ovel, &tpos, &tvel);
  if (behind_run) CMH_CUDA(cudaStreamWaitEvent(side_stream, ev_pos_free, 0));
  for (int i = 0; i < nbox; i++)
    if (parts[i].n > 0)
      CMH_CUDA(cudaMemcpyAsync(in_pos[b].as<unsigned char>() + opos[i], parts[i].pos,
                               (size_t)parts[i].n * 3 * (parts[i].pos_dtype == CMH_FLOAT64 ? 8 : 4),
                               cudaMemcpyHostToDevice, side_stream));
  CMH_CUDA(cudaEventRecord(ev_pos[b], side_stream));
  if (behind_run) CMH_CUDA(cudaStreamWaitEvent(side_stream, ev_vel_free, 0));
  for (int i = 0; i < nbox; i++)
    if (parts[i].n > 0)
      CMH_CUDA(cudaMemcpyAsync(in_vel[b].as<unsigned char>() + ovel[i], parts[i].vel,
                               (size_t)parts[i].n * 3 * (parts[i].vel_dtype == CMH_FLOAT64 ? 8 : 4),
                               cudaMemcpyHostToDevice, side_stream));
  CMH_CUDA(cudaEventRecord(ev_vel[b], side_stream));
}

void Plan::queue_pending() {
  // (a run on device-resident particles records no free events: what is
  // staged waits for the next run on host inputs)
  if (input_buffers != 1 || !vel_wait || staged.empty() || !staged.front().pending) return;
  Staged &f = staged.front();
  std::vector<size_t> opos, ovel;
  size_t tpos, tvel;
  input_layout(f.parts.data(), (int)f.parts.size(), &opos, &ovel, &tpos, &tvel);
  // the buffer is in use by the queued run: it is not grown now (a larger
  // next run is copied when it starts)
  if (tpos > in_pos[0].cap || tvel > in_vel[0].cap) return;
  copy_inputs(f.parts.data(), (int)f.parts.size(), 0, true);
  f.pending = false;
  overwritten = true;
}

std::vector<cmh_particles> Plan::take_inputs(const cmh_particles *parts, int nbox,
                                             cudaStream_t s) {
  int b = -1;
  cur_host.assign(parts, parts + nbox);
  overwritten = false;
  if (!staged.empty()) {
    const Staged &f = staged.front();
    if (same_inputs(f.parts, parts, nbox)) {
      if (!f.pending) b = f.buf;  // else copied now, below
      staged.erase(staged.begin());
    } else {
      // not what was staged: the staged copies are dropped
      CMH_CUDA(cudaStreamSynchronize(side_stream));
      staged.clear();
    }
  }
  // not staged: copied now, into the first buffer (a plan that is never
  // given prefetches keeps a single input buffer)
  if (b < 0) b = stage_inputs(parts, nbox, s, 0);
  last_buf = b;
  CMH_CUDA(cudaStreamWaitEvent(s, ev_pos[b], 0));
  ev_vel_ready = ev_vel[b];
  vel_wait = true;
  std::vector<size_t> opos, ovel;
  size_t tpos, tvel;
  input_layout(parts, nbox, &opos, &ovel, &tpos, &tvel);
  std::vector<cmh_particles> dp(parts, parts + nbox);
  for (int i = 0; i < nbox; i++) {
    dp[i].pos = in_pos[b].as<unsigned char>() + opos[i];
    dp[i].vel = in_vel[b].as<unsigned char>() + ovel[i];
    dp[i].location = CMH_DEVICE;
  }
  return dp;
}

void Plan::run(const cmh_particles &parts, bool want_member, cudaStream_t s) {
  BoxSpec sp;
  sp.params = params;
  sp.ltab = ltab_host;
  sp.pos = parts.pos;
  sp.vel = parts.vel;
  sp.vel_f64 = parts.vel_dtype == CMH_FLOAT64;
  sp.n = parts.n;
  sp.cell_factor = 0;
  run_batch({sp}, want_member, s);
}

}  // namespace cmh
