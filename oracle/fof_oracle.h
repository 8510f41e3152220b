/* CPU restatement of CM_Halofinder's FoF hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the checker for the GPU halo finder.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load it; the product path never does.
 *
 * It restates src_v2/FOF.c of the reference (cell grid FOF.c:45-92, stencil
 * FOF.c:96-161, pair predicate FOF.c:351-357, halo retrieval FOF.c:189-201,
 * Checkhalo FOF.c:378-430, properties FOF.c:797-872) with one change: the
 * ring splice of Befriend (FOF.c:359-373) is replaced by a union-find.  Both
 * compute the connected components of the same pair predicate, so the
 * partition is identical; only the member order inside a halo differs, which
 * changes the floating-point summation order of the halo properties.
 *
 * Parity of this restatement is pinned against the reference itself, built
 * from its own sources by oracle/Makefile (oracle/_ref), on the fixtures in
 * tests/golden/.
 */
#ifndef CMH_FOF_ORACLE_H
#define CMH_FOF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double lo[3], hi[3];   /* Lxmin..Lzmax (startup.c:152-174) */
  double boundary;       /* Boundarysize (startup.c:184) */
  double linklength;     /* Linklength (startup.c:188) */
  double nphalomin;      /* Nphalomin (startup.c:192) */
  int periodic;          /* build images within `boundary` of the faces */
  int pos_is_double;     /* part_datatype: 0 = float (MEMORY_MODE), 1 = double */
  int vel_is_double;
  int cells[3];          /* Px, Py, Pz: lcell = (L + 2b) / P (FOF.c:50-52) */
  int props;             /* bit 0: INERTIA, bit 1: DISPERSION */
  /* variable linking length: ll[i] for cell-centre radius table (0 = off) */
  int varlink;
  double origin[3];
  int ltab_n;            /* entries of a uniform table over r in [0, ltab_rmax] */
  double ltab_rmax;
  const double *ltab;    /* linking length at r = i * ltab_rmax / (ltab_n - 1) */
} cmh_oracle_params;

typedef struct {
  int64_t n_in;          /* particles given */
  int64_t n_out;         /* dropped: outside the domain (read_data.c:409-424) */
  int64_t n_kept;        /* originals kept */
  int64_t n_images;      /* periodic images added */
  int64_t n_proc;        /* n_kept + n_images */
  int64_t n_groups;      /* FoF groups, singletons included */
  int64_t n_candidates;  /* groups with n >= Nphalomin */
  int64_t nhalos;        /* candidates whose centre of mass is owned */
  int64_t n_edge_warn;   /* owned halos with a member within Linklength of
                            the shell edge (the warning of FOF.c:403-422) */
  int64_t n_pair_tests;  /* pair predicate evaluations */
  int64_t n_member_conflicts; /* an input particle in two owned halos */
} cmh_oracle_stats;

/* Number of floats per halo record: n, x, y, z, vx, vy, vz [, 6 inertia]
 * [, 6 dispersion] (FOF.c:574-580). */
int cmh_oracle_halosize(int props);

/* Processing array: kept originals in input order, then periodic images
 * grouped by source particle (input order) and shift code
 * (sz+1)*9 + (sy+1)*3 + (sx+1) ascending.  An image's coordinate is
 * (part_datatype)((double)x + s*(hi-lo)) and it is kept iff every shifted
 * coordinate lies in [lo-b, hi+b].  Outputs may be NULL to count only.
 * Returns the processing count, or -1 on bad arguments. */
int64_t cmh_oracle_build_proc(const cmh_oracle_params *p, int64_t n,
                              const void *pos, uint32_t *proc_src,
                              void *proc_pos, cmh_oracle_stats *st);

/* FoF over a processing array (non-periodic semantics on [lo-b, hi+b]).
 *   group[i]       : lowest processing index of i's group (the ring head)
 *   halo_head[h]   : head of owned halo h, ascending (FOF.c:296-298 order)
 *   halo_props[h*] : the halo record (cmh_oracle_halosize floats)
 *   member[src]    : index of the owned halo holding the particle or one of
 *                    its images, -1 otherwise (n_src entries; may be NULL);
 *                    the lowest index if two owned halos hold copies
 * halo arrays need room for n_proc entries.  Returns 0, or a negative code:
 * -1 bad arguments, -2 Linklength larger than the cell size (the reference
 * would silently miss pairs), -3 a particle outside [lo-b, hi+b]
 * (read_data.c:810-812). */
int cmh_oracle_fof(const cmh_oracle_params *p, int64_t n_proc,
                   const void *proc_pos, const void *proc_vel,
                   const uint32_t *proc_src, int64_t n_src,
                   int64_t *group, uint32_t *halo_head, float *halo_props,
                   int64_t *member, cmh_oracle_stats *st);

/* Squared linking length of fixed-grid cell (ix, iy, iz) under the
 * variable-linking-length rule (see fof_oracle.c). */
double cmh_oracle_cell_linksq(const cmh_oracle_params *p, const double *rmin_buff,
                              const double *lcell, int ix, int iy, int iz);

/* The exact pair predicate of FOF.c:351-357: d2 <= linksq with d2 evaluated
 * as ((dx*dx + dy*dy) + dz*dz) in double, dx = Pos - Pos in part_datatype. */
int cmh_oracle_linked_f32(const float *a, const float *b, double linksq);
int cmh_oracle_linked_f64(const double *a, const double *b, double linksq);

#ifdef __cplusplus
}
#endif
#endif
