/* CPU restatement of CM_Halofinder's FoF hot path -- TEST INFRASTRUCTURE ONLY.
 * See fof_oracle.h for the contract and the reference lines it follows.
 * Built with -ffp-contract=off so that every double expression rounds the
 * way the reference's x86-64 build does (no fused multiply-add).
 */
#include "fof_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

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

static int64_t uf_find(int64_t *parent, int64_t x) {
  while (parent[x] != x) {
    parent[x] = parent[parent[x]];
    x = parent[x];
  }
  return x;
}

static void uf_union(int64_t *parent, int64_t a, int64_t b) {
  a = uf_find(parent, a);
  b = uf_find(parent, b);
  if (a == b) return;
  if (a < b) parent[b] = a;
  else parent[a] = b;
}

int cmh_oracle_fof(const cmh_oracle_params *p, int64_t n_proc,
                   const void *proc_pos, const void *proc_vel,
                   const uint32_t *proc_src, int64_t n_src,
                   int64_t *group, uint32_t *halo_head, float *halo_props,
                   int64_t *member, cmh_oracle_stats *st) {
  if (!p || n_proc < 0 || !group || !halo_head || !halo_props) return -1;
  if (n_proc > 0 && (!proc_pos || !proc_vel)) return -1;
  const int dbl = p->pos_is_double;
  const int vdbl = p->vel_is_double;
  double rmin_buff[3], rmax_buff[3], lcell[3];
  int nc[3];
  for (int a = 0; a < 3; a++) {
    rmin_buff[a] = p->lo[a] - p->boundary;               /* startup.c:40-47 */
    rmax_buff[a] = p->hi[a] + p->boundary;
    if (p->cells[a] <= 0) return -1;
    lcell[a] = (p->hi[a] - p->lo[a] + 2.0 * p->boundary) / p->cells[a]; /* FOF.c:50-52 */
    nc[a] = (int)ceil((rmax_buff[a] - rmin_buff[a]) / lcell[a]) + 1;    /* FOF.c:63-65 */
  }
  double linksq = p->linklength * p->linklength;                        /* FOF.c:60 */
  double maxlink = p->linklength;
  if (p->varlink) {
    if (p->ltab_n < 2 || !p->ltab) return -1;
    maxlink = 0;
    for (int i = 0; i < p->ltab_n; i++)
      if (p->ltab[i] > maxlink) maxlink = p->ltab[i];
  }
  for (int a = 0; a < 3; a++)
    if (maxlink > lcell[a]) return -2;

  const int64_t ncell = (int64_t)nc[0] * nc[1] * nc[2];
  int64_t *first = (int64_t *)malloc(sizeof(int64_t) * (size_t)(ncell > 0 ? ncell : 1));
  int64_t *chain = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_proc + 1));
  int64_t *parent = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_proc + 1));
  if (!first || !chain || !parent) { free(first); free(chain); free(parent); return -1; }
  for (int64_t c = 0; c < ncell; c++) first[c] = -1;

  /* set chain (FOF.c:76-92): head-of-list per cell, LIFO */
  for (int64_t i = 0; i < n_proc; i++) {
    parent[i] = i;
    int ic[3];
    for (int a = 0; a < 3; a++) {
      double x = getpos(proc_pos, dbl, i, a);
      if (x < rmin_buff[a] || x > rmax_buff[a]) {
        free(first); free(chain); free(parent);
        return -3;
      }
      ic[a] = (int)floor((x - rmin_buff[a]) / lcell[a]);
    }
    int64_t ind = ((int64_t)ic[2] * nc[1] + ic[1]) * nc[0] + ic[0];
    chain[i] = first[ind];
    first[ind] = i;
  }

  int64_t ntests = 0;
  for (int iz = 0; iz < nc[2]; iz++)
    for (int iy = 0; iy < nc[1]; iy++)
      for (int ix = 0; ix < nc[0]; ix++) {
        int64_t ip = first[((int64_t)iz * nc[1] + iy) * nc[0] + ix];
        if (ip < 0) continue;
        double lsq = linksq;
        if (p->varlink) lsq = cmh_oracle_cell_linksq(p, rmin_buff, lcell, ix, iy, iz);
        do {
          /* same cell (FOF.c:114-119) */
          for (int64_t ip2 = chain[ip]; ip2 >= 0; ip2 = chain[ip2]) {
            int lk = dbl ? cmh_oracle_linked_f64((const double *)proc_pos + 3 * ip,
                                                 (const double *)proc_pos + 3 * ip2, lsq)
                         : cmh_oracle_linked_f32((const float *)proc_pos + 3 * ip,
                                                 (const float *)proc_pos + 3 * ip2, lsq);
            ntests++;
            if (lk) uf_union(parent, ip, ip2);
          }
          /* 13 forward cells (FOF.c:122-153) */
          for (int iz2 = iz; iz2 <= iz + 1; iz2++) {
            if (iz2 >= nc[2]) continue;
            int iy1 = (iz2 == iz) ? iy : iy - 1;
            for (int iy2 = iy1; iy2 <= iy + 1; iy2++) {
              if (iy2 >= nc[1] || iy2 < 0) continue;
              int ix1 = (iz2 == iz && iy2 == iy) ? ix : ix - 1;
              for (int ix2 = ix1; ix2 <= ix + 1; ix2++) {
                if (ix2 >= nc[0] || ix2 < 0) continue;
                if (ix2 == ix && iy2 == iy && iz2 == iz) continue;
                int64_t ip2 = first[((int64_t)iz2 * nc[1] + iy2) * nc[0] + ix2];
                for (; ip2 >= 0; ip2 = chain[ip2]) {
                  int lk = dbl ? cmh_oracle_linked_f64((const double *)proc_pos + 3 * ip,
                                                       (const double *)proc_pos + 3 * ip2, lsq)
                               : cmh_oracle_linked_f32((const float *)proc_pos + 3 * ip,
                                                       (const float *)proc_pos + 3 * ip2, lsq);
                  ntests++;
                  if (lk) uf_union(parent, ip, ip2);
                }
              }
            }
          }
          ip = chain[ip];
        } while (ip >= 0);
      }
  free(first);

  /* Retrieval.  The union-find root is the lowest index of the group, the
   * same particle the reference's head scan (FOF.c:189-201) calls the head. */
  int64_t *count = chain; /* reuse: count per root */
  for (int64_t i = 0; i < n_proc; i++) count[i] = 0;
  int64_t ngroups = 0;
  for (int64_t i = 0; i < n_proc; i++) {
    int64_t r = uf_find(parent, i);
    group[i] = r;
    if (count[r]++ == 0) ngroups++;
  }
  /* members of each group in ascending index order: bucket lists */
  int64_t *mstart = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_proc + 1));
  int64_t *mlist = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_proc > 0 ? n_proc : 1));
  if (!mstart || !mlist) { free(mstart); free(mlist); free(chain); free(parent); return -1; }
  {
    int64_t acc = 0;
    for (int64_t i = 0; i < n_proc; i++) { mstart[i] = acc; acc += count[i]; }
    mstart[n_proc] = acc;
    int64_t *fill = parent; /* parent no longer needed after group[] */
    for (int64_t i = 0; i < n_proc; i++) fill[i] = mstart[i];
    for (int64_t i = 0; i < n_proc; i++) mlist[fill[group[i]]++] = i;
  }
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
  free(chain);
  free(parent);
  return 0;
}
