/* Single-rank implementations of the MPI and GSL entry points that the
 * reference's src_v2 sources call.  Test infrastructure only: it lets the
 * unmodified reference FOF() run on one core as the oracle's pin.
 *
 * With NTask == 1 every collective is a copy of the rank's own block:
 *   MPI_Alltoall(v)  read_data.c:525,771   -> memcpy of block 0
 *   MPI_Allgather    FOF.c:926-928         -> memcpy of one element
 *   MPI_Reduce       read_data.c:849       -> memcpy
 * The particle exchange uses a derived struct type built from member offsets
 * (read_data.c:722-764); its extent is the end of the last block rounded up
 * to the strictest member alignment, as MPI defines it.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "mpi.h"
#include "gsl/gsl_rng.h"

struct cmh_mpi_type cmh_mpi_int_t = {sizeof(int), sizeof(int)};
struct cmh_mpi_type cmh_mpi_unsigned_t = {sizeof(unsigned), sizeof(unsigned)};
struct cmh_mpi_type cmh_mpi_float_t = {sizeof(float), sizeof(float)};
struct cmh_mpi_type cmh_mpi_double_t = {sizeof(double), sizeof(double)};
struct cmh_mpi_type cmh_mpi_ull_t = {sizeof(unsigned long long),
                                     sizeof(unsigned long long)};

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
int MPI_Abort(MPI_Comm c, int code) { (void)c; fflush(stdout); exit(code); }
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c) {
  (void)buf; (void)count; (void)t; (void)root; (void)c; return 0;
}
int MPI_Alltoall(const void *sbuf, int scount, MPI_Datatype st, void *rbuf,
                 int rcount, MPI_Datatype rt, MPI_Comm c) {
  (void)rcount; (void)rt; (void)c;
  memmove(rbuf, sbuf, (size_t)scount * (size_t)st->extent);
  return 0;
}
int MPI_Alltoallv(const void *sbuf, const int *scounts, const int *sdispls,
                  MPI_Datatype st, void *rbuf, const int *rcounts,
                  const int *rdispls, MPI_Datatype rt, MPI_Comm c) {
  (void)rcounts; (void)c;
  memmove((char *)rbuf + (size_t)rdispls[0] * (size_t)rt->extent,
          (const char *)sbuf + (size_t)sdispls[0] * (size_t)st->extent,
          (size_t)scounts[0] * (size_t)st->extent);
  return 0;
}
int MPI_Allgather(const void *sbuf, int scount, MPI_Datatype st, void *rbuf,
                  int rcount, MPI_Datatype rt, MPI_Comm c) {
  (void)rcount; (void)rt; (void)c;
  memmove(rbuf, sbuf, (size_t)scount * (size_t)st->extent);
  return 0;
}
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t,
               MPI_Op op, int root, MPI_Comm c) {
  (void)op; (void)root; (void)c;
  memmove(rbuf, sbuf, (size_t)count * (size_t)t->extent);
  return 0;
}
int MPI_Get_address(const void *loc, MPI_Aint *addr) {
  *addr = (MPI_Aint)(size_t)loc;
  return 0;
}
int MPI_Type_create_struct(int count, const int *blocklens,
                           const MPI_Aint *displs, const MPI_Datatype *types,
                           MPI_Datatype *newtype) {
  long end = 0, align = 1;
  for (int i = 0; i < count; i++) {
    long e = (long)displs[i] + (long)blocklens[i] * types[i]->extent;
    if (e > end) end = e;
    if (types[i]->align > align) align = types[i]->align;
  }
  struct cmh_mpi_type *t = (struct cmh_mpi_type *)malloc(sizeof *t);
  t->extent = (end + align - 1) / align * align;
  t->align = align;
  *newtype = t;
  return 0;
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }

static const gsl_rng_type cmh_ranlxd1_type = {0};
const gsl_rng_type *gsl_rng_ranlxd1 = &cmh_ranlxd1_type;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t) {
  (void)t;
  return (gsl_rng *)calloc(1, sizeof(gsl_rng));
}
void gsl_rng_set(gsl_rng *r, unsigned long seed) { r->state = seed; }
double gsl_rng_uniform(gsl_rng *r) {
  (void)r;
  fprintf(stderr, "ref harness: subsampling needs GSL's ranlxd1, which is "
                  "not available; run with SampInHalos/SampOutHalos < 0\n");
  abort();
}
void gsl_rng_free(gsl_rng *r) { free(r); }
