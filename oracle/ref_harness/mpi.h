/* Single-rank stand-in for <mpi.h>, test infrastructure only.
 *
 * MPI is not installed in this image.  The reference's src_v2 sources call a
 * small set of MPI routines (main.c:8-10,65,76,110; read_data.c:131,180,525,
 * 547,727-772,822,846,849; startup.c:304; FOF.c:541,910,926-928).  With one
 * rank every collective degenerates to a local copy, which is what
 * ref_stubs.c implements, so the reference FOF() can be compiled and run
 * unmodified as the pinning oracle for the GPU halo finder.
 */
#ifndef CMH_REF_HARNESS_MPI_H
#define CMH_REF_HARNESS_MPI_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct cmh_mpi_type { long extent; long align; } *MPI_Datatype;

extern struct cmh_mpi_type cmh_mpi_int_t, cmh_mpi_unsigned_t, cmh_mpi_float_t,
    cmh_mpi_double_t, cmh_mpi_ull_t;

#define MPI_COMM_WORLD 0
#define MPI_SUM 1
#define MPI_INT (&cmh_mpi_int_t)
#define MPI_UNSIGNED (&cmh_mpi_unsigned_t)
#define MPI_FLOAT (&cmh_mpi_float_t)
#define MPI_DOUBLE (&cmh_mpi_double_t)
#define MPI_UNSIGNED_LONG_LONG (&cmh_mpi_ull_t)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm c, int *rank);
int MPI_Comm_size(MPI_Comm c, int *size);
int MPI_Barrier(MPI_Comm c);
int MPI_Abort(MPI_Comm c, int code);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Alltoall(const void *sbuf, int scount, MPI_Datatype st, void *rbuf,
                 int rcount, MPI_Datatype rt, MPI_Comm c);
int MPI_Alltoallv(const void *sbuf, const int *scounts, const int *sdispls,
                  MPI_Datatype st, void *rbuf, const int *rcounts,
                  const int *rdispls, MPI_Datatype rt, MPI_Comm c);
int MPI_Allgather(const void *sbuf, int scount, MPI_Datatype st, void *rbuf,
                  int rcount, MPI_Datatype rt, MPI_Comm c);
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t,
               MPI_Op op, int root, MPI_Comm c);
int MPI_Get_address(const void *loc, MPI_Aint *addr);
int MPI_Type_create_struct(int count, const int *blocklens,
                           const MPI_Aint *displs, const MPI_Datatype *types,
                           MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *t);

#ifdef __cplusplus
}
#endif
#endif
