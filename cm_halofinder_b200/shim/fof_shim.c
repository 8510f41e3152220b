/* Drop-in replacement of CM_Halofinder's src_v2/FOF.c.
 *
 * The program keeps its own main.c, startup.c, read_data.c and vars.c; this
 * file takes the place of FOF.c and provides the one function main() calls,
 * FOF() (declared vars.h:121, called main.c:73).  FOF() hands the rank's
 * particles P[0 .. nparticles_tot) -- originals and the ghost copies that
 * Read_Data received -- to the B200 halo finder through the C ABI of
 * libcmh_fof, then writes the same files as the reference:
 *   "<OutputFileBase>.<ThisTask>"  the halo catalog (Output_Halos,
 *                                  FOF.c:546-913), with the same -D flags;
 *   "<OutputFileBase>.info"        the task table (Output_Info, FOF.c:917-957);
 *   "<OutputFileBase>_inhalo.<ThisTask>", "..._outhalo.<ThisTask>"
 *                                  the subsamples (Subsample, FOF.c:432-544)
 *                                  when SampInHalos / SampOutHalos > 0.
 * Like the reference, FOF() frees P (FOF.c:333).  Errors go through
 * FatalError (main.c:107-112) after printing the library's message.
 *
 * Build it with the program's own flags (MEMORY_MODE, PARTICLE_ID,
 * OUTPUT_UNFORMATTED, OUTPUT_PARTICLES, INERTIA, DISPERSION) in place of
 * FOF.c, with -I<this repository>/include, and link -lcmh_fof.
 *
 * Subsampling keeps each particle with its group's rate as the reference
 * does, but draws its own uniforms (a hash of Seed and the particle's ID or
 * index) instead of GSL RANLUX numbers along the linked rings, so the sample
 * has the same law, not the same particles.  VARLINK builds stop with an
 * error (the reference's own VARLINK build does not compile).  The domain is
 * the rank's [rmin, rmax) with its ghost shell already in P, so the library
 * runs non-periodic and keeps the halos whose centre of mass the rank owns,
 * as Checkhalo does (FOF.c:378-430).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vars.h"
#include "cmh_fof.h"

static void shim_fatal(const char *what, int line) {
  char msg[1024];
  cmh_last_error(msg, sizeof msg);
  printf("\nERROR: %s: %s\n\n", what, msg);
  fflush(stdout);
  FatalError((char *)"fof_shim.c", line);
}

#ifdef MEMORY_MODE
typedef float shim_real;
#define SHIM_DTYPE CMH_FLOAT32
#else
typedef double shim_real;
#define SHIM_DTYPE CMH_FLOAT64
#endif

void FOF(void) {
  if (cmh_abi_version() != CMH_ABI_VERSION) {
    printf("\nERROR: libcmh_fof has ABI version %d, this program was built for %d; "
           "rebuild it against the library's cmh_fof.h.\n\n",
           cmh_abi_version(), CMH_ABI_VERSION);
    FatalError((char *)"fof_shim.c", __LINE__);
  }
#ifdef VARLINK
  printf("\nERROR: the B200 FOF() does not support VARLINK builds.\n\n");
  FatalError((char *)"fof_shim.c", __LINE__);
#endif

  cmh_fof_params p;
  memset(&p, 0, sizeof p);
  for (int a = 0; a < 3; a++) {
    p.lo[a] = rmin[a];
    p.hi[a] = rmax[a];
  }
  p.boundary = boundarysize;
  p.linklength = linklength;
  p.nphalomin = nphalomin;
  p.periodic = 0;  /* Read_Data has placed the ghost copies in P already */
  p.precision = CMH_FP32_RECHECK;
#ifdef INERTIA
  p.properties |= CMH_PROP_INERTIA;
#endif
#ifdef DISPERSION
  p.properties |= CMH_PROP_DISPERSION;
#endif

  /* struct part_data is an array of structures; the ABI takes interleaved
   * Pos[3] and Vel[3] arrays (and the IDs apart) */
  const size_t n = nparticles_tot;
  shim_real *pos = (shim_real *)malloc(3 * (n ? n : 1) * sizeof(shim_real));
  shim_real *vel = (shim_real *)malloc(3 * (n ? n : 1) * sizeof(shim_real));
  uint64_t *ids = NULL;
  if (!pos || !vel) {
    printf("\nERROR: Task %d cannot allocate the particle copies.\n\n", ThisTask);
    FatalError((char *)"fof_shim.c", __LINE__);
  }
  for (size_t i = 0; i < n; i++)
    for (int a = 0; a < 3; a++) {
      pos[3 * i + a] = P[i].Pos[a];
      vel[3 * i + a] = P[i].Vel[a];
    }
#ifdef PARTICLE_ID
  ids = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
  if (!ids) FatalError((char *)"fof_shim.c", __LINE__);
  for (size_t i = 0; i < n; i++) ids[i] = (uint64_t)P[i].ID;
#endif
  cmh_particles parts;
  memset(&parts, 0, sizeof parts);
  parts.n = (int64_t)n;
  parts.pos_dtype = SHIM_DTYPE;
  parts.vel_dtype = SHIM_DTYPE;
  parts.pos = pos;
  parts.vel = vel;
  parts.id = ids;
  parts.location = CMH_HOST;

  cmh_catalog cat;
  cmh_sample sample;
  memset(&sample, 0, sizeof sample);
  const int sampled = SampInHalos > 0 || SampOutHalos > 0;
  if (sampled) {
    cmh_sampling sp;
    memset(&sp, 0, sizeof sp);
    sp.samp_in = SampInHalos > 0 ? SampInHalos : 0.0;
    sp.samp_out = SampOutHalos > 0 ? SampOutHalos : 0.0;
    sp.seed = Seed;
#ifndef PERIODIC
    /* the last rank along an axis keeps particles on its upper face
       (FOF.c:215-229) */
    sp.closed_hi[0] = Local_nx == Nx - 1;
    sp.closed_hi[1] = Local_ny == Ny - 1;
    sp.closed_hi[2] = Local_nz == Nz - 1;
#endif
    if (cmh_fof_run_sampled(&p, &parts, &sp, &cat, /*want_member=*/1, &sample, NULL) != CMH_OK)
      shim_fatal("FoF on the GPU failed", __LINE__);
  } else if (cmh_fof_run(&p, &parts, &cat, /*want_member=*/1, NULL) != CMH_OK) {
    shim_fatal("FoF on the GPU failed", __LINE__);
  }
  if (cat.stats.n_edge_warn > 0)
    printf("\nWARNING: Task %d has %lld halo(s) within a linking length of its "
           "boundary region; increase Boundarysize.\n\n",
           ThisTask, (long long)cat.stats.n_edge_warn);

  if (ThisTask == 0) {
    printf("Outputting the halos\n");
    printf("====================\n\n");
  }
  unsigned flags = 0;
#ifdef OUTPUT_UNFORMATTED
  flags |= CMH_OUT_UNFORMATTED;
#endif
#ifdef OUTPUT_PARTICLES
  flags |= CMH_OUT_PARTICLES;
#endif
#ifdef PARTICLE_ID
  flags |= CMH_OUT_PARTICLE_ID;
#endif
  if (cmh_write_halos(OutputFileBase, ThisTask, &cat, &parts, flags) != CMH_OK)
    shim_fatal("writing the halo catalog failed", __LINE__);
  /* the subsamples (FOF.c:303-318); no file for an empty one */
  const uint32_t sflags = flags & (CMH_OUT_UNFORMATTED | CMH_OUT_PARTICLE_ID);
  if (SampInHalos > 0 &&
      cmh_write_subsample(OutputFileBase, ThisTask, 1, &parts, sample.inhalo, sample.n_inhalo,
                          sflags) != CMH_OK)
    shim_fatal("writing the in-halo subsample failed", __LINE__);
  if (SampOutHalos > 0 &&
      cmh_write_subsample(OutputFileBase, ThisTask, 0, &parts, sample.outhalo, sample.n_outhalo,
                          sflags) != CMH_OK)
    shim_fatal("writing the out-of-halo subsample failed", __LINE__);

  /* the info file: every task's halo and subsample counts to task 0
     (FOF.c:926-928) */
  int nh = (int)cat.nhalos;
  unsigned nsub[2] = {(unsigned)sample.n_inhalo, (unsigned)sample.n_outhalo};
  int *table = (int *)malloc(sizeof(int) * (size_t)NTask);
  unsigned *subtab = (unsigned *)malloc(2 * sizeof(unsigned) * (size_t)NTask);
  if (!table || !subtab) FatalError((char *)"fof_shim.c", __LINE__);
  MPI_Allgather(&nh, 1, MPI_INT, table, 1, MPI_INT, MPI_COMM_WORLD);
  MPI_Allgather(&nsub[0], 1, MPI_UNSIGNED, subtab, 1, MPI_UNSIGNED, MPI_COMM_WORLD);
  MPI_Allgather(&nsub[1], 1, MPI_UNSIGNED, subtab + NTask, 1, MPI_UNSIGNED, MPI_COMM_WORLD);
  if (ThisTask == 0) {
    cmh_run_parameters rp;
    memset(&rp, 0, sizeof rp);
    rp.Nx = Nx;
    rp.Ny = Ny;
    rp.Nz = Nz;
    rp.Px = Px;
    rp.Py = Py;
    rp.Pz = Pz;
    rp.Lxmin = Lxmin;
    rp.Lymin = Lymin;
    rp.Lzmin = Lzmin;
    rp.Lxmax = Lxmax;
    rp.Lymax = Lymax;
    rp.Lzmax = Lzmax;
    int64_t *counts = (int64_t *)malloc(3 * sizeof(int64_t) * (size_t)NTask);
    if (!counts) FatalError((char *)"fof_shim.c", __LINE__);
    for (int t = 0; t < NTask; t++) {
      counts[t] = table[t];
      counts[NTask + t] = subtab[t];
      counts[2 * NTask + t] = subtab[NTask + t];
    }
    if (cmh_write_info_sampled(OutputFileBase, &rp, counts, counts + NTask, counts + 2 * NTask,
                               NTask) != CMH_OK)
      shim_fatal("writing the info file failed", __LINE__);
    free(counts);
  }
  free(subtab);
  free(table);

  cmh_sample_free(&sample);
  cmh_catalog_free(&cat);
  free(ids);
  free(vel);
  free(pos);
  free(P); /* FOF() owns P from here on, as in the reference (FOF.c:333) */
  P = NULL;
}
