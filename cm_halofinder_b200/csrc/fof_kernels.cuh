// Device-side geometry, pair predicates and union-find of the FoF pipeline.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cmh {

constexpr int kMaxBoxes = 1024;       // domains per run
constexpr int kMaxCellFactor = 32;    // fine cells per top-cell edge

// Particle position in cell order with the index of its source particle.
template <class PT> struct SPos;
template <> struct __align__(16) SPos<float> {
  float x, y, z;
  uint32_t src;
};
template <> struct __align__(16) SPos<double> {
  double x, y, z;
  uint32_t src, pad;
};

// Geometry and run parameters of one domain, passed by value to kernels.
struct Geom {
  double lo[3], hi[3];   // Lmin, Lmax
  double rmin[3];        // lo - boundary (grid origin, rmin_buff)
  double rmax[3];        // hi + boundary (rmax_buff)
  double L[3];           // hi - lo
  double boundary;
  double linksq;         // Linklength^2 in double (FOF.c:60)
  double maxlink;        // largest linking length (edge warning, pruning)
  double prune_sq;       // (maxlink * (1 + 1e-5))^2: pairs of cells farther apart never link
  double h;              // fine cell side, <= minimum linking length / sqrt(3)
  double inv_h;          // 1 / h
  double nphalomin;
  float t_lo, t_hi;      // FP32 band: d2 < t_lo links, d2 > t_hi does not
  int periodic;
  int k;                 // fine cells per top-cell edge
  int W;                 // fine-cell reach: cells more than W apart never link
  int G[3];              // fine cells per axis
  int T[3];              // top cells per axis
  uint64_t k3;           // k^3
  uint32_t kmul;         // floor(2^32 / k) + 1: x / k == umulhi(x, kmul) for x < 2^27
  int props;             // CMH_PROP_* bits
  int hs;                // floats per halo record
  uint32_t union_cap;    // retries of a union before it gives up (the plan's limit)
  // variable linking length
  int varlink;
  double origin[3];
  double ref_lcell[3];   // fixed grid of the l(r) rule
  int ref_nc[3];
  int ltab_n;
  double ltab_dr;
  const double *ltab;    // device copy of the table
};

// One domain of a run (a run holds one or many), in device memory.
struct BoxDev {
  Geom g;
  const void *pos;      // n x 3, the plan's position dtype
  const void *vel;      // n x 3
  uint64_t in_base;     // first index of the box in the run's input numbering
  uint64_t top_base;    // first index of the box's top cells in the run's tables
  uint32_t n;           // input particles of the box
  int vel_f64;          // velocities are double
};

// Device-side sizes of one run: nothing is read back by the host until the
// run has been issued, so the whole run can be captured in a CUDA graph.
struct DevScal {
  uint32_t kept_total, img_total;  // totals of the keep / image scans
  uint32_t np_raw, np;             // processed particles (np clamped to the capacity)
  uint32_t R, nd, nc, nh;          // fine cells, dense top cells, candidates, halos
  uint32_t qcount, next_dense, next0, next1;
  uint32_t overflow;               // bit 0: processed particles above capacity
  uint32_t nbig, next_big;          // dense top cells handled by a whole CTA
  uint32_t next_simple;             // fine cells taken by the sparse path
  uint32_t failed;                  // a sort's capped look-back wait gave up: every
                                    // later kernel of the run returns at once
};

// Running counters of one run, in device memory.
struct Counters {
  unsigned long long pair_tests;
  unsigned long long rechecks;
  unsigned long long member_conflicts;
  unsigned int uf_giveups;     // union loops that hit their iteration cap
  unsigned int domain_errors;  // particles outside [rmin, rmax] after ingest
  unsigned long long cand_pairs;   // fine-cell pairs within reach
  unsigned long long root_skips;   // ... already in one component
  unsigned long long unions;       // ... joined by a linked particle pair
  unsigned long long find_steps;   // parent loads in the befriending finds
  unsigned long long scan_iters;   // fine cells scanned in sparse top cells
  unsigned long long window_iters; // map slots visited in dense top cells
  unsigned int sort_giveups;       // radix-sort look-back waits that hit their cap
};

// FP32 band around l^2: returns the thresholds t_lo < fl32(l2) < t_hi such
// that d2_32 < t_lo implies the double test links and d2_32 > t_hi implies
// it does not (proof in fof.cu above band_thresholds()).
__host__ __device__ inline void band_thresholds(double l2, int ulps, float *t_lo,
                                                float *t_hi) {
  float l2f = (float)l2;
  int e;
  frexp((double)l2f, &e);                       // l2f in [2^(e-1), 2^e)
  double ulp = ldexp(1.0, e - 1 - 23);          // spacing of floats at l2f
  double lo = (double)l2f - ulps * ulp;
  double hi = (double)l2f + ulps * ulp;
  // outward rounding to float keeps the band at least this wide
  float flo = (float)lo, fhi = (float)hi;
  if ((double)flo > lo) flo = nextafterf(flo, -INFINITY);
  if ((double)fhi < hi) fhi = nextafterf(fhi, INFINITY);
  *t_lo = flo;
  *t_hi = fhi;
}

// ---- variable linking length (one value per cell of a fixed grid) ----
//
// The reference gives every cell of its fixed grid (Px x Py x Pz cells of
// side lcell over the padded domain, FOF.c:45-52) one linking length, looked
// up at the cell's distance from the observer (link.c:1-13,
// FOF.c:102-109), and tests a pair with the length of the cell its scan
// starts from: the lower of the two cells in (z, y, x) order, since each
// cell scans itself and its 13 forward neighbours (FOF.c:111-153).  Pairs
// whose cells are not neighbours are never tested.  Each processed particle
// therefore carries its grid cell (packed z << 42 | y << 21 | x, which
// orders like the scan) and that cell's l^2; the FP32 form derives its band
// from that l^2 (vl_band below).
struct __align__(16) VLRec64 {
  uint64_t rkey;
  double lsq;
};
template <bool FP32> using VLRec = VLRec64;

// The FP32 band around a variable l^2 from the bits of fl32(l^2): from
// 2 ulps steps below to ulps steps above.  A step below fl32(l^2) is at
// least half its spacing (less only across a power of two), so the band
// holds at least `ulps` spacings on each side -- the band of
// band_thresholds(), which is the one the proof needs.  A subnormal or zero
// fl32(l^2) sends every pair to the double test.
__device__ __forceinline__ void vl_band(double lsq, int ulps, float *t_lo, float *t_hi) {
  const uint32_t b = __float_as_uint(__double2float_rn(lsq));
  if (b < 0x00800000u) {
    *t_lo = -1.0f;
    *t_hi = __int_as_float(0x7f800000);
    return;
  }
  *t_lo = __uint_as_float(b - 2u * (uint32_t)ulps);
  *t_hi = __uint_as_float(b + (uint32_t)ulps);
}

// Cell of the fixed grid holding (x, y, z): floor((x - rmin_buff) / lcell)
// per axis, in double with IEEE division (FOF.c:76-92).
__device__ __forceinline__ uint64_t ref_key(const Geom &g, double x, double y, double z) {
  const double c[3] = {x, y, z};
  uint64_t key = 0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    int i = (int)floor(__ddiv_rn(__dsub_rn(c[a], g.rmin[a]), g.ref_lcell[a]));
    i = i < 0 ? 0 : (i > (1 << 21) - 1 ? (1 << 21) - 1 : i);
    key |= (uint64_t)i << (21 * a);
  }
  return key;
}

// l^2 of a grid cell: the table l(r) (ltab_n values on r = 0, dr, ...,
// rmax, linear in between, the last value beyond) at the distance of the
// cell centre from the observer; every operation rounded as written.
__device__ __forceinline__ double ref_cell_linksq(const Geom &g, uint64_t rkey) {
  double q = 0.0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double i = (double)(int)((rkey >> (21 * a)) & 0x1fffffull);
    const double c = __dadd_rn(__dsub_rn(g.rmin[a], g.origin[a]),
                               __dmul_rn(__dadd_rn(i, 0.5), g.ref_lcell[a]));
    q = a == 0 ? __dmul_rn(c, c) : __dadd_rn(q, __dmul_rn(c, c));
  }
  const double t = __ddiv_rn(__dsqrt_rn(q), g.ltab_dr);
  double l;
  if (t >= (double)(g.ltab_n - 1)) {
    l = g.ltab[g.ltab_n - 1];
  } else {
    const int i = (int)t;
    const double f = __dsub_rn(t, (double)i);
    l = __dadd_rn(__dmul_rn(g.ltab[i], __dsub_rn(1.0, f)), __dmul_rn(g.ltab[i + 1], f));
  }
  return __dmul_rn(l, l);
}

// Whether two grid cells are equal or neighbours (|difference| <= 1 per axis).
__device__ __forceinline__ bool ref_neighbours(uint64_t a, uint64_t b) {
  bool ok = true;
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const int d = (int)((a >> (21 * s)) & 0x1fffffull) - (int)((b >> (21 * s)) & 0x1fffffull);
    ok &= d >= -1 && d <= 1;
  }
  return ok;
}

// x / k for a fine-cell coordinate x < 2^21 (2 <= k <= 32): with kmul =
// floor(2^32 / k) + 1 = (2^32 + e) / k, 0 < e <= k, x kmul / 2^32 = x / k +
// x e / (k 2^32), and the second term stays below 1/k, so the floor is exact.
__device__ __forceinline__ int div_k(int x, const Geom &g) {
  return (int)__umulhi((uint32_t)x, g.kmul);
}

// Fine-cell index along one axis: floor((x - rmin) * (1/h)), in double.  Two
// points with the same index are within h (1 + 4e-16 * index) of each other
// along the axis, far inside the 2^-20 margin that sizes h.
__device__ __forceinline__ int fine_index(double x, double rmin, double inv_h, int G) {
  double q = __dmul_rn(__dsub_rn(x, rmin), inv_h);
  int g = (int)floor(q);
  g = g < 0 ? 0 : g;
  return g >= G ? G - 1 : g;
}

// ---- union-find over occupied fine cells (lock-free, hook to min root) ----
//
// parent[x] <= x always holds: a root is only ever hooked under a smaller
// root (atomicCAS), and path halving only stores ancestors.  Chains are
// therefore strictly decreasing and find() terminates; the final root of a
// component is its smallest cell index.

__device__ __forceinline__ uint32_t uf_find(uint32_t *parent, uint32_t x) {
  while (true) {
    uint32_t p = __ldcg(parent + x);
    if (p == x) return x;
    uint32_t gp = __ldcg(parent + p);
    if (gp == p) return p;
    __stcg(parent + x, gp);  // path halving: gp is an ancestor of x
    x = gp;
  }
}

// find() that also counts its parent loads
__device__ __forceinline__ uint32_t uf_find_n(uint32_t *parent, uint32_t x,
                                              unsigned long long &steps) {
  while (true) {
    uint32_t p = __ldcg(parent + x);
    steps++;
    if (p == x) return x;
    uint32_t gp = __ldcg(parent + p);
    steps++;
    if (gp == p) return p;
    __stcg(parent + x, gp);
    x = gp;
  }
}

constexpr uint32_t kUnionCap = 1u << 22;  // default retries of a union

// Joins the components of a and b; retries after a lost race at most `cap`
// times, then counts a give-up (the run reports CMH_ERR_DEVICE_TIMEOUT;
// parents stay valid cell indices, so nothing downstream leaves its bounds).
__device__ __forceinline__ void uf_union(uint32_t *parent, uint32_t a, uint32_t b,
                                         Counters *ctr, uint32_t cap = kUnionCap) {
  for (uint32_t it = 0; it < cap; it++) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return;
    if (a < b) {
      uint32_t t = a;
      a = b;
      b = t;
    }
    // hook the larger root a under the smaller root b
    uint32_t old = atomicCAS(parent + a, a, b);
    if (old == a) return;
    a = old;  // a was hooked meanwhile; retry from its new parent
  }
  atomicAdd(&ctr->uf_giveups, 1u);
}

}  // namespace cmh
