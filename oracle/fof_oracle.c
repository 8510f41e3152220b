/* CPU restatement of CM_Halofinder's FoF hot path -- TEST INFRASTRUCTURE ONLY.
 * See fof_oracle.h for the contract and the reference lines it follows.
 * Built with -ffp-contract=off so that every double expression rounds the
 * way the reference's x86-64 build does (no fused multiply-add).
 */
#include "fof_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

int cmh_oracle_halosize(int props) {
  int hs = 7;                 /* FOF.c:574 */
  if (props & 1) hs += 6;     /* INERTIA, FOF.c:575-577 */
  if (props & 2) hs += 6;     /* DISPERSION, FOF.c:578-580 */
  return hs;
}

static inline double getpos(const void *pos, int is_double, int64_t i, int a) {
  return is_double ? ((const double *)pos)[3 * i + a]
                   : (double)((const float *)pos)[3 * i + a];
}

/* ---------------------------------------------------------------------- */
/* Processing array (ingest + periodic images).                            */
/* ---------------------------------------------------------------------- */

/* read_data.c:409-424: a particle is outside iff x < xmin || x > xmax, with
 * the domain widened by Boundarysize in non-periodic runs.  A NaN coordinate
 * is treated as outside (the reference would index a cell with it). */
static int inside(const cmh_oracle_params *p, double x, int a) {
  double lo = p->lo[a], hi = p->hi[a];
  if (!p->periodic) {
    lo -= p->boundary;
    hi += p->boundary;
  }
  return x >= lo && x <= hi;
}

int64_t cmh_oracle_build_proc(const cmh_oracle_params *p, int64_t n,
                              const void *pos, uint32_t *proc_src,
                              void *proc_pos, cmh_oracle_stats *st) {
  if (!p || n < 0 || (n > 0 && !pos)) return -1;
  const int dbl = p->pos_is_double;
  int64_t m = 0, nout = 0;
  for (int64_t i = 0; i < n; i++) {
    int ok = 1;
    for (int a = 0; a < 3; a++) ok &= inside(p, getpos(pos, dbl, i, a), a);
    if (!ok) { nout++; continue; }
    if (proc_src) proc_src[m] = (uint32_t)i;
    if (proc_pos) {
      for (int a = 0; a < 3; a++) {
        if (dbl) ((double *)proc_pos)[3 * m + a] = ((const double *)pos)[3 * i + a];
        else ((float *)proc_pos)[3 * m + a] = ((const float *)pos)[3 * i + a];
      }
    }
    m++;
  }
  const int64_t nkept = m;
  if (p->periodic) {
    /* Images: the wrap of read_data.c:792-797 applied to a single domain.
     * For Lmin = 0 the reference's rmin - ((Lmax-Lmin) - x) and rmax + x
     * equal x - L and x + L exactly, which is what is computed here. */
    for (int64_t i = 0; i < n; i++) {
      double x[3];
      int ok = 1;
      for (int a = 0; a < 3; a++) {
        x[a] = getpos(pos, dbl, i, a);
        ok &= inside(p, x[a], a);
      }
      if (!ok) continue;
      for (int code = 0; code < 27; code++) {
        if (code == 13) continue;
        int s[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
        double c[3];
        int keep = 1;
        for (int a = 0; a < 3 && keep; a++) {
          if (s[a] == 0) { c[a] = x[a]; continue; }
          double L = p->hi[a] - p->lo[a];
          double v = x[a] + (double)s[a] * L;
          double stored = dbl ? v : (double)(float)v;
          if (stored < p->lo[a] - p->boundary || stored > p->hi[a] + p->boundary)
            keep = 0;
          c[a] = stored;
        }
        if (!keep) continue;
        if (proc_src) proc_src[m] = (uint32_t)i;
        if (proc_pos) {
          for (int a = 0; a < 3; a++) {
            if (dbl) ((double *)proc_pos)[3 * m + a] = c[a];
            else ((float *)proc_pos)[3 * m + a] = (float)c[a];
          }
        }
        m++;
      }
    }
  }
  if (st) {
    st->n_in = n;
    st->n_out = nout;
    st->n_kept = nkept;
    st->n_images = m - nkept;
    st->n_proc = m;
  }
  return m;
}

/* ---------------------------------------------------------------------- */
/* Pair predicate (FOF.c:351-357).                                         */
/* ---------------------------------------------------------------------- */

int cmh_oracle_linked_f32(const float *a, const float *b, double linksq) {
  /* dx is a float subtraction in MEMORY_MODE, widened to double. */
  double dx = (double)(float)(a[0] - b[0]);
  double dy = (double)(float)(a[1] - b[1]);
  double dz = (double)(float)(a[2] - b[2]);
  double d2 = dx * dx + dy * dy + dz * dz;
  return !(d2 > linksq);
}

int cmh_oracle_linked_f64(const double *a, const double *b, double linksq) {
  double dx = a[0] - b[0];
  double dy = a[1] - b[1];
  double dz = a[2] - b[2];
  double d2 = dx * dx + dy * dy + dz * dz;
  return !(d2 > linksq);
}

/* ---------------------------------------------------------------------- */
/* Variable linking length: one value per scanning cell.                   */
/* ---------------------------------------------------------------------- */

/* The linking length of a cell of the fixed grid, at the cell centre.  This
 * is the per-cell rule the reference intends (link.c:1-4, FOF.c:102-109)
 * with the (ix-0.5) offset of FOF.c:105 read as (ix+0.5) like the other two
 * axes, and the table lookup that FOF.c:108 discards actually used. */
double cmh_oracle_cell_linksq(const cmh_oracle_params *p, const double *rmin_buff,
                              const double *lcell, int ix, int iy, int iz) {
  double cx = rmin_buff[0] - p->origin[0] + ((double)ix + 0.5) * lcell[0];
  double cy = rmin_buff[1] - p->origin[1] + ((double)iy + 0.5) * lcell[1];
  double cz = rmin_buff[2] - p->origin[2] + ((double)iz + 0.5) * lcell[2];
  double r = sqrt(cx * cx + cy * cy + cz * cz);
  double dr = p->ltab_rmax / (double)(p->ltab_n - 1);
  double t = r / dr;
  double l;
  if (t >= (double)(p->ltab_n - 1)) {
    l = p->ltab[p->ltab_n - 1];
  } else {
    int i = (int)t;
    double f = t - (double)i;
    l = p->ltab[i] * (1.0 - f) + p->ltab[i + 1] * f;
  }
  return l * l;
}

/* ---------------------------------------------------------------------- */
/* FoF (FOF.c:23-161 with union-find in place of Befriend's ring splice).  */
/* ---------------------------------------------------------------------- */

/* Union-find over cell-ordered slots (see below), hook to the lower slot. */
static uint32_t uf_find(uint32_t *parent, uint32_t x) {
  while (parent[x] != x) {
    parent[x] = parent[parent[x]];
    x = parent[x];
  }
  return x;
}

/* Joins the components of roots a != b; returns the new root. */
static uint32_t uf_hook(uint32_t *parent, uint32_t a, uint32_t b) {
  if (a < b) { parent[b] = a; return a; }
  parent[a] = b;
  return b;
}

typedef struct { uint32_t a, b; } link_t;

/* What the cell scan shares between threads (read-only) and keeps per thread. */
typedef struct {
  const cmh_oracle_params *p;
  int dbl, nc[3];
  const int64_t *cstart;          /* first slot of every cell, ncell + 1 */
  const void *spos;               /* positions in slot order */
  double rmin_buff[3], lcell[3], linksq;
  _Atomic int64_t *next_row;      /* rows (iz, iy) handed out one at a time */
} scan_shared;

typedef struct {
  const scan_shared *sh;
  uint32_t *parent;               /* this thread's union-find over all slots */
  link_t *links;                  /* the joins it made: a spanning forest of its links */
  int64_t nlinks, caplinks, ntests;
  int err;
} scan_thread;

static void add_link(scan_thread *t, uint32_t a, uint32_t b) {
  if (t->nlinks == t->caplinks) {
    int64_t cap = t->caplinks ? 2 * t->caplinks : 4096;
    link_t *nl = (link_t *)realloc(t->links, sizeof(link_t) * (size_t)cap);
    if (!nl) { t->err = 1; return; }
    t->links = nl;
    t->caplinks = cap;
  }
  t->links[t->nlinks].a = a;
  t->links[t->nlinks].b = b;
  t->nlinks++;
}

/* Slot i against slots [j0, j1): the pair predicate for every j not already
 * in i's component.  Skipping a pair whose two particles are already
 * connected leaves the connected components -- the partition -- unchanged. */
static void scan_range(scan_thread *t, uint32_t i, int64_t j0, int64_t j1, double lsq) {
  const scan_shared *sh = t->sh;
  uint32_t *parent = t->parent;
  uint32_t ri = uf_find(parent, i);
  for (int64_t j = j0; j < j1; j++) {
    uint32_t rj = uf_find(parent, (uint32_t)j);
    if (rj == ri) continue;
    int lk = sh->dbl ? cmh_oracle_linked_f64((const double *)sh->spos + 3 * i,
                                             (const double *)sh->spos + 3 * j, lsq)
                     : cmh_oracle_linked_f32((const float *)sh->spos + 3 * i,
                                             (const float *)sh->spos + 3 * j, lsq);
    t->ntests++;
    if (lk) {
      add_link(t, i, (uint32_t)j);
      ri = uf_hook(parent, ri, rj);
    }
  }
}

/* The cell loop of FOF.c:96-161 over one row (iz, iy) of cells: each particle
 * of a cell against the later particles of the same cell (FOF.c:114-119) and
 * every particle of the 13 forward cells (FOF.c:122-153), so that each
 * unordered cell pair is visited once. */
static void scan_row(scan_thread *t, int iz, int iy) {
  const scan_shared *sh = t->sh;
  const int *nc = sh->nc;
  for (int ix = 0; ix < nc[0]; ix++) {
    const int64_t c = ((int64_t)iz * nc[1] + iy) * nc[0] + ix;
    const int64_t a0 = sh->cstart[c], a1 = sh->cstart[c + 1];
    if (a0 == a1) continue;
    double lsq = sh->linksq;
    if (sh->p->varlink)
      lsq = cmh_oracle_cell_linksq(sh->p, sh->rmin_buff, sh->lcell, ix, iy, iz);
    for (int64_t i = a0; i < a1; i++) {
      scan_range(t, (uint32_t)i, i + 1, a1, lsq);
      for (int iz2 = iz; iz2 <= iz + 1; iz2++) {
        if (iz2 >= nc[2]) continue;
        int iy1 = (iz2 == iz) ? iy : iy - 1;
        for (int iy2 = iy1; iy2 <= iy + 1; iy2++) {
          if (iy2 >= nc[1] || iy2 < 0) continue;
          int ix1 = (iz2 == iz && iy2 == iy) ? ix : ix - 1;
          for (int ix2 = ix1; ix2 <= ix + 1; ix2++) {
            if (ix2 >= nc[0] || ix2 < 0) continue;
            if (ix2 == ix && iy2 == iy && iz2 == iz) continue;
            const int64_t c2 = ((int64_t)iz2 * nc[1] + iy2) * nc[0] + ix2;
            scan_range(t, (uint32_t)i, sh->cstart[c2], sh->cstart[c2 + 1], lsq);
          }
        }
      }
    }
  }
}

static void *scan_worker(void *arg) {
  scan_thread *t = (scan_thread *)arg;
  const scan_shared *sh = t->sh;
  const int64_t nrows = (int64_t)sh->nc[2] * sh->nc[1];
  while (!t->err) {
    int64_t r = atomic_fetch_add(sh->next_row, 1);
    if (r >= nrows) break;
    scan_row(t, (int)(r / sh->nc[1]), (int)(r % sh->nc[1]));
  }
  return NULL;
}

/* Threads of the cell scan: CMH_ORACLE_THREADS, else the online cores; one
 * for small inputs. */
static int scan_threads(int64_t n_proc) {
  if (n_proc < 200000) return 1;
  const char *e = getenv("CMH_ORACLE_THREADS");
  long t = e ? strtol(e, NULL, 10) : sysconf(_SC_NPROCESSORS_ONLN);
  if (t < 1) t = 1;
  if (t > 64) t = 64;
  return (int)t;
}

int cmh_oracle_fof(const cmh_oracle_params *p, int64_t n_proc,
                   const void *proc_pos, const void *proc_vel,
                   const uint32_t *proc_src, int64_t n_src,
                   int64_t *group, uint32_t *halo_head, float *halo_props,
                   int64_t *member, cmh_oracle_stats *st) {
  if (!p || n_proc < 0 || !group || !halo_head || !halo_props) return -1;
  if (n_proc > 0 && (!proc_pos || !proc_vel)) return -1;
  if (n_proc >= (int64_t)0xffffffffll) return -1;
  const int dbl = p->pos_is_double;
  const int vdbl = p->vel_is_double;
  scan_shared sh;
  memset(&sh, 0, sizeof sh);
  sh.p = p;
  sh.dbl = dbl;
  double *rmin_buff = sh.rmin_buff, rmax_buff[3], *lcell = sh.lcell;
  int *nc = sh.nc;
  for (int a = 0; a < 3; a++) {
    rmin_buff[a] = p->lo[a] - p->boundary;               /* startup.c:40-47 */
    rmax_buff[a] = p->hi[a] + p->boundary;
    if (p->cells[a] <= 0) return -1;
    lcell[a] = (p->hi[a] - p->lo[a] + 2.0 * p->boundary) / p->cells[a]; /* FOF.c:50-52 */
    nc[a] = (int)ceil((rmax_buff[a] - rmin_buff[a]) / lcell[a]) + 1;    /* FOF.c:63-65 */
  }
  sh.linksq = p->linklength * p->linklength;                            /* FOF.c:60 */
  double maxlink = p->linklength;
  if (p->varlink) {
    if (p->ltab_n < 2 || !p->ltab) return -1;
    maxlink = 0;
    for (int i = 0; i < p->ltab_n; i++)
      if (p->ltab[i] > maxlink) maxlink = p->ltab[i];
  }
  for (int a = 0; a < 3; a++)
    if (maxlink > lcell[a]) return -2;

  /* Cell of every particle (FOF.c:76-92).  The reference chains each cell's
   * particles into a linked list; here they are counting-sorted into slots,
   * each cell's particles contiguous and in ascending index order.  The
   * order in which pairs are tested does not change the components. */
  const int64_t ncell = (int64_t)nc[0] * nc[1] * nc[2];
  const size_t pw = dbl ? sizeof(double) : sizeof(float);
  int64_t *cell = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_proc > 0 ? n_proc : 1));
  int64_t *cstart = (int64_t *)calloc((size_t)ncell + 2, sizeof(int64_t));
  uint32_t *slot_src = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n_proc > 0 ? n_proc : 1));
  void *spos = malloc(3 * pw * (size_t)(n_proc > 0 ? n_proc : 1));
  if (!cell || !cstart || !slot_src || !spos) {
    free(cell); free(cstart); free(slot_src); free(spos);
    return -1;
  }
  for (int64_t i = 0; i < n_proc; i++) {
    int ic[3];
    for (int a = 0; a < 3; a++) {
      double x = getpos(proc_pos, dbl, i, a);
      if (!(x >= rmin_buff[a] && x <= rmax_buff[a])) {
        free(cell); free(cstart); free(slot_src); free(spos);
        return -3;
      }
      ic[a] = (int)floor((x - rmin_buff[a]) / lcell[a]);
    }
    cell[i] = ((int64_t)ic[2] * nc[1] + ic[1]) * nc[0] + ic[0];
    cstart[cell[i] + 1]++;
  }
  for (int64_t c = 0; c < ncell; c++) cstart[c + 1] += cstart[c];
  {
    /* cstart[c] walks from the start to the end of cell c, then the starts
     * are shifted back */
    for (int64_t i = 0; i < n_proc; i++) {
      const int64_t k = cstart[cell[i]]++;
      slot_src[k] = (uint32_t)i;
      memcpy((char *)spos + 3 * pw * (size_t)k, (const char *)proc_pos + 3 * pw * (size_t)i, 3 * pw);
    }
    for (int64_t c = ncell; c > 0; c--) cstart[c] = cstart[c - 1];
    cstart[0] = 0;
  }
  free(cell);
  sh.cstart = cstart;
  sh.spos = spos;

  /* The scan, rows of cells spread over threads.  Each thread keeps its own
   * union-find and records the joins it makes (a spanning forest of the
   * links it found); the forests of all threads span the same components as
   * all links together, and are merged below. */
  const int nt = scan_threads(n_proc);
  _Atomic int64_t next_row = 0;
  sh.next_row = &next_row;
  scan_thread *th = (scan_thread *)calloc((size_t)nt, sizeof(scan_thread));
  uint32_t *parent = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n_proc > 0 ? n_proc : 1));
  int err = !th || !parent;
  for (int k = 0; k < nt && !err; k++) {
    th[k].sh = &sh;
    th[k].parent = k == 0 ? parent : (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n_proc > 0 ? n_proc : 1));
    if (!th[k].parent) { err = 1; break; }
    for (int64_t i = 0; i < n_proc; i++) th[k].parent[i] = (uint32_t)i;
  }
  if (!err) {
    if (nt == 1) {
      scan_worker(&th[0]);
    } else {
      pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
      int started = 0;
      if (!tid) err = 1;
      for (int k = 0; k < nt && !err; k++) {
        if (pthread_create(&tid[k], NULL, scan_worker, &th[k]) != 0) { err = 1; break; }
        started++;
      }
      for (int k = 0; k < started; k++) pthread_join(tid[k], NULL);
      free(tid);
    }
  }
  int64_t ntests = 0;
  if (!err) {
    /* thread 0's union-find already holds its own joins; add the others' */
    for (int k = 1; k < nt; k++)
      for (int64_t q = 0; q < th[k].nlinks; q++) {
        uint32_t ra = uf_find(parent, th[k].links[q].a), rb = uf_find(parent, th[k].links[q].b);
        if (ra != rb) uf_hook(parent, ra, rb);
      }
    for (int k = 0; k < nt; k++) {
      ntests += th[k].ntests;
      err |= th[k].err;
    }
  }
  for (int k = 0; th && k < nt; k++) {
    if (k > 0) free(th[k].parent);
    free(th[k].links);
  }
  free(th);
  free(cstart);
  free(spos);
  if (err) { free(parent); free(slot_src); return -1; }

  /* Retrieval.  The reference's head (FOF.c:189-201) is the lowest index of
   * the group: per component the lowest particle index of its slots. */
  int64_t *count = (int64_t *)calloc((size_t)(n_proc > 0 ? n_proc : 1), sizeof(int64_t));
  uint32_t *low = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n_proc > 0 ? n_proc : 1));
  if (!count || !low) { free(count); free(low); free(parent); free(slot_src); return -1; }
  for (int64_t k = 0; k < n_proc; k++) low[k] = 0xffffffffu;
  for (int64_t k = 0; k < n_proc; k++) {
    const uint32_t r = uf_find(parent, (uint32_t)k);
    if (slot_src[k] < low[r]) low[r] = slot_src[k];
  }
  int64_t ngroups = 0;
  for (int64_t k = 0; k < n_proc; k++) {
    const int64_t h = low[uf_find(parent, (uint32_t)k)];
    group[slot_src[k]] = h;
    if (count[h]++ == 0) ngroups++;
  }
  free(low);
  free(parent);
  free(slot_src);
  /* members of each group in ascending index order: bucket lists */
  int64_t *mstart = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_proc + 1));
  int64_t *mlist = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_proc > 0 ? n_proc : 1));
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_proc > 0 ? n_proc : 1));
  if (!mstart || !mlist || !fill) { free(mstart); free(mlist); free(fill); free(count); return -1; }
  {
    int64_t acc = 0;
    for (int64_t i = 0; i < n_proc; i++) { mstart[i] = acc; acc += count[i]; }
    mstart[n_proc] = acc;
    for (int64_t i = 0; i < n_proc; i++) fill[i] = mstart[i];
    for (int64_t i = 0; i < n_proc; i++) mlist[fill[group[i]]++] = i;
  }
  free(fill);
  if (member)
    for (int64_t s = 0; s < n_src; s++) member[s] = -1;

  const int hs = cmh_oracle_halosize(p->props);
  int64_t ncand = 0, nh = 0, nwarn = 0, nconf = 0;
  for (int64_t i = 0; i < n_proc; i++) {
    if (group[i] != i) continue;
    int64_t n = count[i];
    if ((double)n < p->nphalomin) continue;          /* FOF.c:202 */
    ncand++;
    const int64_t *mem = mlist + mstart[i];
    /* Checkhalo (FOF.c:378-401): centre of mass by division */
    double xh = 0, yh = 0, zh = 0;
    for (int64_t k = 0; k < n; k++) {
      xh += getpos(proc_pos, dbl, mem[k], 0);
      yh += getpos(proc_pos, dbl, mem[k], 1);
      zh += getpos(proc_pos, dbl, mem[k], 2);
    }
    xh /= (double)n;
    yh /= (double)n;
    zh /= (double)n;
    if (xh < p->lo[0] || xh >= p->hi[0]) continue;
    if (yh < p->lo[1] || yh >= p->hi[1]) continue;
    if (zh < p->lo[2] || zh >= p->hi[2]) continue;
    /* edge warning (FOF.c:406-422) */
    int warn = 0;
    for (int64_t k = 0; k < n && !warn; k++)
      for (int a = 0; a < 3; a++) {
        double x = getpos(proc_pos, dbl, mem[k], a);
        if (x - rmin_buff[a] < maxlink || rmax_buff[a] - x < maxlink) warn = 1;
      }
    nwarn += warn;
    /* Output_Halos (FOF.c:797-872): sums in double, means by the reciprocal */
    double inv = 1.0 / (double)n;
    double s[6] = {0, 0, 0, 0, 0, 0};
    double xx = 0, yy = 0, zz = 0, xy = 0, xz = 0, yz = 0;
    double vxx = 0, vyy = 0, vzz = 0, vxy = 0, vxz = 0, vyz = 0;
    for (int64_t k = 0; k < n; k++) {
      double x = getpos(proc_pos, dbl, mem[k], 0);
      double y = getpos(proc_pos, dbl, mem[k], 1);
      double z = getpos(proc_pos, dbl, mem[k], 2);
      double vx = getpos(proc_vel, vdbl, mem[k], 0);
      double vy = getpos(proc_vel, vdbl, mem[k], 1);
      double vz = getpos(proc_vel, vdbl, mem[k], 2);
      s[0] += x; s[1] += y; s[2] += z;
      s[3] += vx; s[4] += vy; s[5] += vz;
      xx += x * x; yy += y * y; zz += z * z;
      xy += x * y; xz += x * z; yz += y * z;
      vxx += vx * vx; vyy += vy * vy; vzz += vz * vz;
      vxy += vx * vy; vxz += vx * vz; vyz += vy * vz;
    }
    float *rec = halo_props + (size_t)nh * hs;
    int o = 0;
    rec[o++] = (float)n;
    for (int k = 0; k < 6; k++) rec[o++] = (float)(s[k] * inv);
    if (p->props & 1) {                                  /* FOF.c:849-854 */
      rec[o++] = (float)(yy + zz - inv * (s[1] * s[1] + s[2] * s[2]));
      rec[o++] = (float)(xx + zz - inv * (s[0] * s[0] + s[2] * s[2]));
      rec[o++] = (float)(xx + yy - inv * (s[0] * s[0] + s[1] * s[1]));
      rec[o++] = (float)(inv * s[0] * s[1] - xy);
      rec[o++] = (float)(inv * s[0] * s[2] - xz);
      rec[o++] = (float)(inv * s[1] * s[2] - yz);
    }
    if (p->props & 2) {                                  /* FOF.c:856-861 */
      rec[o++] = (float)((vxx - s[3] * s[3] * inv) * inv);
      rec[o++] = (float)((vyy - s[4] * s[4] * inv) * inv);
      rec[o++] = (float)((vzz - s[5] * s[5] * inv) * inv);
      rec[o++] = (float)((vxy - s[3] * s[4] * inv) * inv);
      rec[o++] = (float)((vxz - s[3] * s[5] * inv) * inv);
      rec[o++] = (float)((vyz - s[4] * s[5] * inv) * inv);
    }
    halo_head[nh] = (uint32_t)i;
    if (member && proc_src) {
      for (int64_t k = 0; k < n; k++) {
        int64_t sidx = proc_src[mem[k]];
        if (sidx < 0 || sidx >= n_src) continue;
        /* a particle in two owned halos (a halo wider than the shell, the
         * case FOF.c:403-422 warns about) keeps the lower catalog index */
        if (member[sidx] < 0) member[sidx] = nh;
        else if (member[sidx] != nh) nconf++;
      }
    }
    nh++;
  }
  if (st) {
    st->n_groups = ngroups;
    st->n_candidates = ncand;
    st->nhalos = nh;
    st->n_edge_warn = nwarn;
    st->n_pair_tests = ntests;
    st->n_member_conflicts = nconf;
  }
  free(mstart);
  free(mlist);
  free(count);
  return 0;
}
