/*
 * mpi.h -- minimal multi-process MPI stand-in used to build and run the
 * reference's own C sources on a machine without MPI.  TEST INFRASTRUCTURE:
 * it exists only so that the reference can serve as the oracle's pin and as
 * the timed CPU baseline.
 *
 * Ranks are forked processes connected pairwise by socketpairs.  Point-to-point
 * messages between a pair are FIFO (tags are not used for matching; the
 * reference's calls are symmetric, so program order matches them).
 * Collectives run through rank 0 in ascending rank order.
 *
 * Environment:
 *   LBRB_SHIM_NP    number of ranks (default 1)
 *   LBRB_SHIM_DIMS  "AxB" overrides MPI_Dims_create for 2-D grids (a test
 *                   hook; a conforming MPI returns non-increasing dims)
 */
#ifndef LBRB_SHIM_MPI_H
#define LBRB_SHIM_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_SUM 1
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_INTEGER 3
#define MPI_CHAR 4
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Dims_create(int nnodes, int ndims, int dims[]);
int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[], int reorder,
                    MPI_Comm *cart);
int MPI_Cart_sub(MPI_Comm cart, const int remain_dims[], MPI_Comm *sub);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype);
int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype old,
                    MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Gatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                const int recvcounts[], const int displs[], MPI_Datatype recvtype, int root,
                MPI_Comm comm);
int MPI_Scatterv(const void *sendbuf, const int sendcounts[], const int displs[],
                 MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype,
                 int root, MPI_Comm comm);
double MPI_Wtime(void);

#endif
