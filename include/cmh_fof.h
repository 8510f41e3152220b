/* cmh_fof.h -- C ABI of the B200 Friends-of-Friends halo finder.
 *
 * Drop-in for the FoF hot path of CM_Halofinder (src_v2/FOF.c, src_v2/link.c).
 * Plain C types only: pointers, sizes and enums.  Every entry point returns a
 * cmh_status; nothing aborts the process (the reference's FatalError ->
 * MPI_Abort, main.c:107-112, becomes a status code plus cmh_last_error()).
 *
 * Threading: a cmh_plan is used by one host thread at a time and issues all
 * device work on the stream given to it.  cmh_last_error() is per thread.
 */
#ifndef CMH_FOF_H
#define CMH_FOF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Bumped whenever a structure's layout or an entry point's signature changes;
 * a caller compares cmh_abi_version() with the value it was built against. */
#define CMH_ABI_VERSION 2

typedef enum cmh_status {
  CMH_OK = 0,
  CMH_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, bad enum          */
  CMH_ERR_PARAMETER_FILE = 2,   /* Read_Parameterfile failures, startup.c:286-306 */
  CMH_ERR_CUDA = 3,             /* a CUDA runtime call failed                */
  CMH_ERR_OUT_OF_MEMORY = 4,    /* device or host allocation failed          */
  CMH_ERR_DOMAIN = 5,           /* particle outside the padded domain
                                   (read_data.c:810-812)                      */
  CMH_ERR_CAPACITY = 6,         /* beyond 32-bit indices, a plan's capacity,
                                   or a fixed scratch area                   */
  CMH_ERR_DEVICE_TIMEOUT = 7,   /* a bounded device loop gave up             */
  CMH_ERR_IO = 8,               /* file could not be opened / written        */
  CMH_ERR_NO_DEVICE = 9         /* no usable sm_100 device                   */
} cmh_status;

typedef enum cmh_dtype { CMH_FLOAT32 = 0, CMH_FLOAT64 = 1 } cmh_dtype;

/* Pair-test arithmetic.  Both give the reference's membership exactly.
 *   CMH_PLAIN_FP64   : every pair test is the reference's double expression
 *                      ((dx*dx + dy*dy) + dz*dz) <= Linklength^2 (FOF.c:351-357)
 *   CMH_FP32_RECHECK : the test runs in FP32; a pair whose FP32 d^2 lies within
 *                      4 ulp (8 ulp for FP64 positions) of FP32(l^2) is
 *                      re-tested with the double expression.                */
typedef enum cmh_precision { CMH_PLAIN_FP64 = 0, CMH_FP32_RECHECK = 1 } cmh_precision;

typedef enum cmh_location { CMH_HOST = 0, CMH_DEVICE = 1 } cmh_location;

#define CMH_PROP_INERTIA 1u    /* -DINERTIA    (FOF.c:849-854) */
#define CMH_PROP_DISPERSION 2u /* -DDISPERSION (FOF.c:856-861) */

/* Run parameters of the hot path: the subset of the reference's globals that
 * FOF() reads (vars.h:100-117), for one domain (Nx = Ny = Nz = 1). */
typedef struct cmh_fof_params {
  double lo[3];        /* Lxmin, Lymin, Lzmin                                 */
  double hi[3];        /* Lxmax, Lymax, Lzmax                                 */
  double boundary;     /* Boundarysize: ghost-shell width                     */
  double linklength;   /* Linklength (upper bound of l(r) when varlink)       */
  double nphalomin;    /* Nphalomin: groups with fewer members are dropped    */
  int32_t periodic;    /* 1: images within `boundary` of the faces are added  */
  int32_t precision;   /* cmh_precision                                       */
  uint32_t properties; /* CMH_PROP_* bits                                     */
  int32_t cell_factor; /* fine cells per top-cell edge, 0 = autotune          */
  /* Variable linking length (link.c): the linking length of a pair is the
   * value at the centre of the lower-index cell of a fixed grid of
   * ref_cells[a] cells over [lo-b, hi+b] (the reference's lcell grid), read
   * from a uniform table over r = |centre - origin| in [0, ltab_rmax].      */
  int32_t varlink;
  int32_t ref_cells[3];
  double origin[3];
  int32_t ltab_n;
  double ltab_rmax;
  const double *ltab;  /* host pointer, ltab_n entries                         */
} cmh_fof_params;

/* Caller-owned particles, the fields of struct part_data (vars.h:36-47) as
 * interleaved arrays: pos[3*i + a], vel[3*i + a]. */
typedef struct cmh_particles {
  int64_t n;
  int32_t pos_dtype;   /* cmh_dtype                                           */
  int32_t vel_dtype;   /* cmh_dtype                                           */
  const void *pos;
  const void *vel;
  const uint64_t *id;  /* optional (PARTICLE_ID), may be NULL                 */
  int32_t location;    /* cmh_location of all three pointers                  */
} cmh_particles;

typedef struct cmh_stats {
  int64_t n_in;            /* particles given                                 */
  int64_t n_out;           /* dropped outside the domain (read_data.c:409-424) */
  int64_t n_images;        /* periodic images added                           */
  int64_t n_proc;          /* particles processed = kept + images             */
  int64_t n_cells;         /* occupied fine cells                             */
  int64_t n_groups;        /* FoF groups, singletons included                 */
  int64_t n_candidates;    /* groups with at least Nphalomin members          */
  int64_t nhalos;          /* candidates whose centre of mass is owned        */
  int64_t n_edge_warn;     /* owned halos with a member within Linklength of
                              the padded-domain edge (FOF.c:403-422)          */
  int64_t n_pair_tests;    /* pair predicate evaluations                      */
  int64_t n_rechecks;      /* FP64 re-tests of band pairs                     */
  int64_t n_member_conflicts; /* particles found in two owned halos           */
  int32_t cell_factor;     /* fine cells per top-cell edge used               */
  int32_t key_bits;        /* significant bits of the sort key                */
  float ms_total;          /* device time of the run (CUDA events)            */
  float stage_ms[8];       /* ingest, sort, cells, befriend, groups, sums,
                              catalog, members (CUDA events on the stream)    */
  int32_t n_launches;      /* kernels launched by the run                     */
  int64_t n_cell_pairs;    /* fine-cell pairs within linking reach            */
  int64_t n_root_skips;    /* ... found already joined                        */
  int64_t n_unions;        /* ... joined by a linked particle pair            */
  int64_t n_find_steps;    /* union-find parent loads while befriending       */
  int64_t n_scan_iters;    /* fine cells scanned in sparse top cells          */
  int64_t n_window_iters;  /* window slots visited in dense top cells         */
  int64_t n_dense_tops;    /* top cells joined in shared memory (dense)       */
  int64_t n_queued;        /* fine cells sent to the warp-per-cell path       */
  int64_t n_big_tops;      /* dense top cells joined by a whole CTA           */
} cmh_stats;

/* Halo catalog in the layout of the reference's unformatted records
 * (FOF.c:836-872): per halo `halosize` floats
 *   n, x, y, z, vx, vy, vz [, Ixx Iyy Izz Ixy Ixz Iyz] [, sxx syy szz sxy sxz syz]
 * in ascending order of the halo head, the lowest processing index of the
 * group (FOF.c:296-298). */
typedef struct cmh_catalog {
  int64_t nhalos;
  int32_t halosize;
  int32_t location;    /* cmh_location of the arrays                          */
  float *props;        /* nhalos * halosize                                   */
  uint32_t *head;      /* nhalos: processing index of the head                */
  int64_t *member;     /* n_in: owned-halo index of each particle (or of one
                          of its images), -1 if none; NULL if not requested   */
  uint32_t *member_proc; /* n_in: processing index of that member copy       */
  float *member_pos;   /* n_in x 3: its coordinates as stored (an image's
                          coordinates are the wrapped ones, as the reference
                          writes them, FOF.c:719-724)                          */
  cmh_stats stats;
  void *impl;          /* library-owned storage                               */
} cmh_catalog;

typedef struct cmh_plan cmh_plan;

/* ---- library ------------------------------------------------------------ */

int cmh_abi_version(void);

/* Message of the last failing call on this host thread. */
size_t cmh_last_error(char *buf, size_t len);

/* Fault injection for tests (host side only, no GPU fault): the environment
 * variable CMH_FAULT holds comma-separated words, read on every call --
 *   alloc    : a device allocation fails (CMH_ERR_OUT_OF_MEMORY)
 *   io       : opening an input or output file fails (CMH_ERR_IO), as the
 *              reference's file helpers stop the run (main.c:83-112)
 *   overflow : every run outgrows its buffers until the plan gives up
 *              (CMH_ERR_CAPACITY), as a rank's receive-buffer overflow stops
 *              the reference (read_data.c:551-556)
 *   lookback : one tile of the cell sort publishes nothing, so that the next
 *              tile's wait runs into its bound (CMH_ERR_DEVICE_TIMEOUT)   */

/* ---- one-shot run: replaces void FOF(void) (src_v2/FOF.c:23, vars.h:121) - */

/* Runs FoF on one domain and fills `cat` (host arrays, freed by
 * cmh_catalog_free).  Particles may be host or device resident.  `want_member`
 * requests cat->member.  `stream` is a cudaStream_t (NULL: legacy stream).
 * Replaces FOF() from the cell grid (FOF.c:45-92) through Checkhalo
 * (FOF.c:378-430) and the property sums of Output_Halos (FOF.c:797-872);
 * the writers are cmh_write_halos / cmh_write_info below. */
cmh_status cmh_fof_run(const cmh_fof_params *params, const cmh_particles *parts,
                       cmh_catalog *cat, int32_t want_member, void *stream);

/* Frees what cmh_fof_run / cmh_plan_run put in a catalog. */
void cmh_catalog_free(cmh_catalog *cat);

/* ---- plans: device-resident repeated runs (same FOF() replacement) ------ */

/* Creates a plan for up to `max_particles` input particles of `pos_dtype`
 * on CUDA device `device`.  Device workspace is allocated here and grown on
 * demand by cmh_plan_run. */
cmh_status cmh_plan_create(cmh_plan **plan, const cmh_fof_params *params,
                           int64_t max_particles, int32_t pos_dtype, int32_t device);

/* Runs FoF on the particles (host-resident ones are first copied into
 * plan-owned device memory on `stream`).  With out_location == CMH_DEVICE
 * the catalog arrays stay in plan-owned device memory (valid until the next
 * run or cmh_plan_destroy); with CMH_HOST they are copied to host arrays that
 * cmh_catalog_free releases. */
cmh_status cmh_plan_run(cmh_plan *plan, const cmh_particles *parts,
                        cmh_catalog *cat, int32_t want_member,
                        int32_t out_location, void *stream);

/* Starts copying host-resident particles (parts->location == CMH_HOST) into
 * plan-owned device memory on a stream of the plan's own, after the work
 * already queued on `stream`, so that the copy overlaps whatever the GPU is
 * doing -- typically the previous run.  A later cmh_plan_run given the same
 * host arrays (same pointers, count and dtypes) uses the staged copy instead
 * of copying again; a run given other host arrays drops what was staged.  At
 * most two runs can be staged ahead (CMH_ERR_INVALID_ARGUMENT beyond).  The
 * host arrays must stay unchanged until that run returns, and be pinned for
 * the copy to overlap.  Without a prefetch, cmh_plan_run copies host inputs
 * itself the same way: positions first, the velocities while the run's first
 * stages go on.  The reference reads its particles before FOF() (Read_Data,
 * read_data.c:100-404); nothing there overlaps. */
cmh_status cmh_plan_prefetch(cmh_plan *plan, const cmh_particles *parts, void *stream);

/* Device buffers for host-resident inputs: 2 (the default) lets
 * cmh_plan_prefetch copy the next run's inputs while the current run still
 * reads its own; with 1 (for workspaces that leave no room for a second copy)
 * the next run's positions are copied into the same buffer once the current
 * run's ingest has read its positions, and its velocities once the property
 * sums have read the velocities, so the copies still overlap most of the
 * run.  Staged copies are dropped.  No reference counterpart. */
cmh_status cmh_plan_set_input_buffers(cmh_plan *plan, int32_t n);

/* cmh_plan_prefetch for the `nbox` host-resident boxes of a later
 * cmh_plan_run_batch (or cmh_plan_run_batch_status) given the same boxes in
 * the same order: every box's positions are copied before any velocities.
 * No reference counterpart (the reference runs one domain per rank). */
cmh_status cmh_plan_prefetch_batch(cmh_plan *plan, const cmh_particles *parts, int32_t nbox,
                                   void *stream);

/* Changes the run parameters of a plan (same precision of positions). */
cmh_status cmh_plan_set_params(cmh_plan *plan, const cmh_fof_params *params);

/* A plan records the launches of a run in a CUDA graph and replays the graph
 * when the next run has the same shape (same particle pointers and counts,
 * parameters and capacities).  `enable` = 0 issues every run eagerly. */
cmh_status cmh_plan_set_graph(cmh_plan *plan, int32_t enable);

/* Autotuner: times runs of these boxes (device-resident, as for
 * cmh_plan_run_batch) over a grid of cell-size scales (fine cells per
 * top-cell edge relative to one particle per top cell) and dense-top
 * thresholds, `repeats` timed runs each, and keeps the fastest setting in
 * the plan for its later runs.  Boxes whose params set cell_factor keep it. */
typedef struct cmh_tuning {
  double cell_scale;   /* chosen scale of the cell-size factor            */
  int32_t dense_min;   /* occupied fine cells above which a top cell is dense */
  float ms;            /* best run time (CUDA events)                     */
  int32_t tried;       /* settings timed                                  */
} cmh_tuning;

cmh_status cmh_plan_autotune(cmh_plan *plan, const cmh_fof_params *params,
                             const cmh_particles *parts, int32_t nbox, int32_t repeats,
                             void *stream, cmh_tuning *out);

/* Applies a setting found earlier (cell_scale > 0, dense_min >= 1) to a
 * plan without timing anything; ms and tried are ignored. */
cmh_status cmh_plan_set_tuning(cmh_plan *plan, const cmh_tuning *tuning);

/* cmh_fof_run_batch on a plan: repeated batches of the same shape replay one
 * CUDA graph.  Any box's error fails the whole call.  The boxes may also be
 * all host-resident: they are then copied into plan-owned device memory as
 * for cmh_plan_run (or taken from cmh_plan_prefetch_batch). */
cmh_status cmh_plan_run_batch(cmh_plan *plan, const cmh_fof_params *params,
                              const cmh_particles *parts, int32_t nbox, cmh_catalog *cats,
                              void *stream);

/* cmh_plan_run_batch with a status per box, so that one bad box does not
 * fail the others: each box's parameters and particle description are
 * checked on their own (box_status[b] = the error, cats[b] left empty), and
 * the boxes that pass run together as one batch.  Returns CMH_OK when that
 * batch ran (or no box passed); if the batch itself fails, every box in it
 * gets the batch's status, which is also returned.  The reference's FOF()
 * stops the whole run on any error (FatalError, main.c:107-112). */
cmh_status cmh_plan_run_batch_status(cmh_plan *plan, const cmh_fof_params *params,
                                     const cmh_particles *parts, int32_t nbox,
                                     cmh_catalog *cats, cmh_status *box_status, void *stream);

/* Bounds of the device loops that retry or wait.  A union of two
 * union-find components (find both roots, hook one under the other) is
 * attempted at most union_attempts times -- it is attempted again only after
 * losing a race to another thread -- and a tile of a radix sort polls a lower
 * tile's state at most lookback_polls times after its first read.  A loop
 * that runs out makes the run return CMH_ERR_DEVICE_TIMEOUT (the plan stays
 * usable; the next run starts afresh).  Negative: the default, 2^22 each.
 * union_attempts = 0 makes every union give up at once (a test setting).
 * The reference has no such loops (one CPU thread per rank). */
typedef struct cmh_limits {
  int64_t union_attempts;
  int64_t lookback_polls;
} cmh_limits;

cmh_status cmh_plan_set_limits(cmh_plan *plan, const cmh_limits *limits);

void cmh_plan_destroy(cmh_plan *plan);

/* ---- batched boxes: many independent domains in one launch sequence ----- */

/* Runs `nbox` independent domains; box b uses params[b] and parts[b]
 * (device-resident, same dtypes for all boxes).  The boxes' particles are
 * processed together: one sort, one befriending pass and one reduction for
 * the whole batch.  cats[b] receives box b's catalog (host arrays); its
 * stats n_in, n_out, n_images, n_proc and nhalos are box b's, the other
 * stats (cells, pair tests, stage times, launches) cover the whole run. */
cmh_status cmh_fof_run_batch(const cmh_fof_params *params, const cmh_particles *parts,
                             int32_t nbox, cmh_catalog *cats, void *stream);

/* ---- allocation-free labels for small sets ------------------------------ */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (a framework already holds nearly all of it, allocation is banned
 * after start-up, or a plugin host lends out only its own buffers): FoF group
 * labels with no cudaMalloc/cudaFree and no allocating library call.  Its
 * scratch is a fixed array in the library's device memory (about 1.5 MB on
 * every GPU that loads the library, held until exit).
 *   pos   : device array, n x 3 of pos_dtype, all inside [lo-b, hi+b]
 *           (otherwise CMH_ERR_DOMAIN)
 *   label : device array, n entries; label[i] = lowest index of i's group,
 *           groups being the connected components of the reference's pair
 *           predicate in double (FOF.c:351-357)
 * Limits: n <= 65536 (CMH_ERR_CAPACITY beyond), non-periodic, constant
 * linking length.  The first call on a device looks up the array's address
 * with that device current; make that first call before any stream capture.
 * All calls share the array: calls whose work overlaps on the GPU race.
 * Returns after the stream has finished the work. */
cmh_status cmh_fof_labels_noalloc(const cmh_fof_params *params, const void *pos,
                                  int32_t pos_dtype, int64_t n, uint32_t *label,
                                  void *stream);

/* ---- subsampling (FOF.c:205-284; files by Subsample, FOF.c:432-544) ---- */

/* SampInHalos / SampOutHalos / Seed.  Each original particle inside the
 * domain ([lo, hi) per axis, [lo, hi] on the axes flagged in closed_hi: the
 * reference closes the upper face of the last rank along an axis in isolated
 * builds, FOF.c:215-229) is kept with the rate of its group:
 * samp_in for groups of at least Nphalomin processed particles (images
 * included), samp_out for the others.  It is kept when u(Seed, key) < rate,
 * key = its ID (or its input index without IDs), u = the top 53 bits of
 * SplitMix64's output mix (Steele, Lea & Flood 2014) of
 * key ^ (Seed * 0xD1B54A32D192ED03), times 2^-53.  The reference draws GSL
 * RANLUX numbers along its linked rings (and stops a ring at its first
 * selected particle outside the domain); neither GSL nor the ring order
 * exists here, so the sample has the same law, not the same particles. */
typedef struct cmh_sampling {
  double samp_in;      /* SampInHalos  (0: none)                              */
  double samp_out;     /* SampOutHalos (0: none)                              */
  int32_t seed;        /* Seed                                                */
  int32_t closed_hi[3];/* 1: the domain includes its upper face on this axis  */
} cmh_sampling;

typedef struct cmh_sample {
  int64_t n_inhalo;    /* kept particles of groups with >= Nphalomin members  */
  int64_t *inhalo;     /* their input indices, ascending (host)               */
  int64_t n_outhalo;   /* kept particles of the other groups                  */
  int64_t *outhalo;
} cmh_sample;

/* cmh_fof_run that also draws the subsample (host arrays in *sample, freed
 * by cmh_sample_free). */
cmh_status cmh_fof_run_sampled(const cmh_fof_params *params, const cmh_particles *parts,
                               const cmh_sampling *sampling, cmh_catalog *cat,
                               int32_t want_member, cmh_sample *sample, void *stream);
void cmh_sample_free(cmh_sample *sample);

/* Writes "<base>_inhalo.<task>" (in != 0) or "<base>_outhalo.<task>" in the
 * layout of Subsample (FOF.c:432-544): unformatted, a count record, then all
 * positions, all velocities and (CMH_OUT_PARTICLE_ID) all IDs, each one
 * record; otherwise one "[ID] x y z vx vy vz" line per particle.  No file for
 * an empty sample.  idx are input indices into the host particles `parts`. */
cmh_status cmh_write_subsample(const char *base, int32_t task, int32_t in,
                               const cmh_particles *parts, const int64_t *idx, int64_t n,
                               uint32_t flags);

/* ---- run-parameter file (startup.c:109-314) ----------------------------- */

/* The reference's tag/value run_parameters file.  Same tags, same rules:
 * `%` starts a comment line, an unknown or repeated tag is an error, every
 * tag must be present (startup.c:258-306).  `build_flags` selects the tags of
 * optional builds: CMH_TAGS_VARLINK adds Omega and Origin_* (startup.c:240-256;
 * Origin_* read as floating point here, the reference's INT typo is not
 * kept), CMH_TAGS_INFOFILE adds InputInfoFile (LIGHTCONE + UNFORMATTED,
 * startup.c:232-238). */
#define CMH_TAGS_VARLINK 1
#define CMH_TAGS_INFOFILE 2
typedef struct cmh_run_parameters {
  int32_t Nx, Ny, Nz, Px, Py, Pz;
  double Lxmin, Lymin, Lzmin, Lxmax, Lymax, Lzmax;
  int32_t Seed;
  double Buffer, Boundarysize, Linklength, Nphalomin, SampInHalos, SampOutHalos;
  int32_t InputStyle, Ninputfiles, Starting_file, Nread, Nwrite;
  char InputFileBase[500];
  char OutputFileBase[500];
  double Omega, Origin_x, Origin_y, Origin_z;
  char InputInfoFile[500];
} cmh_run_parameters;

cmh_status cmh_read_parameterfile(const char *fname, int32_t build_flags,
                                  cmh_run_parameters *out);

/* FoF parameters of one rank's domain from the run parameters, as
 * Set_Params derives rmin/rmax (startup.c:33-47) for rank `task` of
 * Nx*Ny*Nz. */
cmh_status cmh_params_from_run(const cmh_run_parameters *rp, int32_t task,
                               int32_t periodic, cmh_fof_params *out);

/* ---- particle readers (read_data.c:100-404) ----------------------------- */

#define CMH_FMT_ASCII 0             /* "[ID] x y z vx vy vz" lines (read_data.c:276-315, 368-404) */
#define CMH_FMT_GADGET1 1           /* -DGADGET_STYLE snapshots (read_data.c:321-365)            */
#define CMH_FMT_PICOLA_LIGHTCONE 2  /* -DLIGHTCONE -DUNFORMATTED files (read_data.c:212-273)     */
#define CMH_READ_PARTICLE_ID 1u     /* -DPARTICLE_ID: the files carry IDs                        */
#define CMH_READ_FP64 2u            /* no MEMORY_MODE: values kept (ASCII: read) as double       */

typedef struct cmh_particle_store cmh_particle_store;

/* Reads every input file of a run, in the reference's order: InputStyle 0
 * reads "<InputFileBase>.<n>" for n = Starting_file .. Starting_file +
 * Ninputfiles - 1, otherwise InputFileBase lists the files (read_data.c:
 * 100-124, 178-198).  The particles of all files are appended in file order
 * into host arrays that *store owns (free with cmh_particle_store_free); the
 * domain filter and ghost images are left to the FoF run, which applies
 * them as Read_Data does.  A missing or short file is CMH_ERR_IO. */
cmh_status cmh_read_particles(const cmh_run_parameters *rp, int32_t format, uint32_t flags,
                              cmh_particles *out, cmh_particle_store **store);
void cmh_particle_store_free(cmh_particle_store *store);

/* ---- catalog writers (FOF.c:546-957) ------------------------------------ */

#define CMH_OUT_UNFORMATTED 1u /* -DOUTPUT_UNFORMATTED */
#define CMH_OUT_PARTICLES 2u   /* -DOUTPUT_PARTICLES   */
#define CMH_OUT_PARTICLE_ID 4u /* -DPARTICLE_ID        */

/* Writes "<base>.<task>" in the reference's layout (Output_Halos,
 * FOF.c:546-913); no file when there are no halos, as there.  With
 * CMH_OUT_PARTICLES the members of each halo follow its record, head first
 * then in ascending processing order (the reference walks its ring from the
 * head); `cat` must carry member, member_proc and member_pos (host) and
 * `parts` (host) supplies velocities and, with CMH_OUT_PARTICLE_ID, IDs. */
cmh_status cmh_write_halos(const char *base, int32_t task, const cmh_catalog *cat,
                           const cmh_particles *parts, uint32_t flags);

/* Writes "<base>.info" (Output_Info, FOF.c:917-957) for one task grid. */
cmh_status cmh_write_info(const char *base, const cmh_run_parameters *rp,
                          const int64_t *nhalos_per_task, int32_t ntask);
/* The same with each task's subsample counts (NSUBSAMPIN, NSUBSAMPOUT);
 * NULL count arrays write zeros. */
cmh_status cmh_write_info_sampled(const char *base, const cmh_run_parameters *rp,
                                  const int64_t *nhalos_per_task,
                                  const int64_t *ninhalo_per_task,
                                  const int64_t *nouthalo_per_task, int32_t ntask);

#ifdef __cplusplus
}
#endif
#endif /* CMH_FOF_H */
