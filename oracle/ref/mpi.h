/*
 * Single-rank MPI stand-in used ONLY to compile the reference PIC3D sources
 * (src/field.cpp, src/particle.cpp, src/boundary.cpp, src/mpi_utils.cpp,
 * src/simulation.cpp) into a CPU oracle binary.  It is test infrastructure,
 * not part of the GPU product.
 *
 * Semantics (one process, rank 0):
 *  - MPI_Cart_shift returns rank 0 (self) for a periodic dimension and
 *    MPI_PROC_NULL (-2, OpenMPI's value, which the reference hard-codes in
 *    mpi_utils.cpp:16-50) otherwise.
 *  - Derived datatypes (contiguous / vector / resized) are flattened to a
 *    list of byte offsets and packed eagerly when MPI_Isend is called.
 *  - A send is delivered immediately if a receive with the same tag is
 *    already posted, otherwise it is queued; MPI_Irecv first looks for a
 *    queued send with its tag.  This is the matching order of a self
 *    transport, so the X, Y and Z halo stages in mpi_utils.cpp complete in
 *    posting order.
 */
#ifndef PIC3D_ORACLE_MPI_SHIM_H
#define PIC3D_ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_BYTE 3
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods,
                    int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *src, int *dst);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allgather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf,
                  int rcount, MPI_Datatype rtype, MPI_Comm comm);

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *out);
int MPI_Type_vector(int count, int blocklen, int stride, MPI_Datatype old,
                    MPI_Datatype *out);
int MPI_Type_create_resized(MPI_Datatype old, long lb, long extent,
                            MPI_Datatype *out);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);

#ifdef __cplusplus
}
#endif

#endif
