/*
 * mpi.h -- single-rank stand-in for the MPI interface, test infrastructure.
 *
 * It lets the reference's own unmodified sources (src/forward/*.cu,
 * src/lib/*.cu, src/media/*.cpp of hpc-lee/gpu-CGFD3D-dynamic) compile and
 * run as one process on one GPU, so that the reference's arithmetic can be
 * compared with the oracle and with this project's CUDA path on identical
 * inputs.  Only the calls the reference makes are declared (gd_t.cu,
 * mympi_t.cu, blk_t.cu, par_t.cu, io_funcs.cu, main_curv_col_el_3d.cu).
 *
 * Semantics for a world of one rank: rank 0 of size 1; the Cartesian
 * topology has no neighbours (MPI_PROC_NULL on every side, as the reference
 * expects on the outer faces of its decomposition); collectives copy the
 * send buffer to the receive buffer; persistent point-to-point requests and
 * their Start/Wait are no-ops because every partner is MPI_PROC_NULL; a
 * point-to-point call with a real partner aborts.  Nothing here is linked
 * into the solver library.
 */
#ifndef CGFD_REFSHIM_MPI_H
#define CGFD_REFSHIM_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
/* a datatype is its size in bytes, so that sizeof(MPI_FLOAT) (used by the
 * reference to size float buffers, blk_t.cu:258) and the copies below are
 * exact for the predefined types */
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS        0
#define MPI_COMM_WORLD     1
#define MPI_PROC_NULL      (-2)
#define MPI_CHAR           1
#define MPI_INT            4
#define MPI_FLOAT          4
#define MPI_REAL           4
#define MPI_LONG           8
#define MPI_DOUBLE         8
#define MPI_MAX            1
#define MPI_MIN            2
#define MPI_SUM            3
#define MPI_STATUS_IGNORE   ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm);
int MPI_Cart_create(MPI_Comm comm, int ndims, const int dims[], const int periods[], int reorder,
                    MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]);
int MPI_Cart_shift(MPI_Comm comm, int dir, int disp, int *source, int *dest);
int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype old, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Send_init(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
                  MPI_Request *req);
int MPI_Recv_init(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
                  MPI_Request *req);
int MPI_Startall(int count, MPI_Request reqs[]);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status *statuses);
int MPI_Sendrecv(const void *sendbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *recvbuf, int rcount, MPI_Datatype rtype, int source, int rtag,
                 MPI_Comm comm, MPI_Status *status);

#ifdef __cplusplus
}
#endif
#endif /* CGFD_REFSHIM_MPI_H */
