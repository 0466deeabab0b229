/*
 * MPI shim -- TEST INFRASTRUCTURE ONLY.
 *
 * Lets the SemiImplicitFV reference sources (C++17 + MPI) compile and run
 * in a container that has no MPI library, so that the reference itself can
 * serve as the parity oracle and as the timed CPU baseline.  Only the
 * symbols the reference calls are provided.
 *
 * By default the process is ONE rank:
 *   - MPI_Cart_shift returns rank 0 (self) for periodic directions and
 *     MPI_PROC_NULL otherwise, as a 1x1x1 Cartesian topology would
 *     (src/MPIContext.cpp:138-140 relies on this);
 *   - MPI_Isend / MPI_Irecv to self are matched by tag in MPI_Waitall
 *     (the periodic self-exchange of src/HaloExchange.cpp:387-408);
 *   - reductions and gathers copy the single contribution.
 *
 * sifv_mpi_shim_run(nranks, fn, user) runs fn(user, rank) on nranks
 * threads that form MPI_COMM_WORLD together (the reference keeps no
 * mutable static state, so its objects of every rank live in one
 * process): MPI_Dims_create factorises as evenly as possible, Cartesian
 * ranks are row-major with no reordering, sends are buffered copies,
 * receives match (source, tag) in order, and reductions combine the
 * contributions in rank order.  It returns when every rank has returned.
 */
#ifndef SIFV_MPI_SHIM_H
#define SIFV_MPI_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL   (-1)
#define MPI_COMM_WORLD  0
#define MPI_COMM_SELF   1
#define MPI_PROC_NULL   (-2)
#define MPI_DOUBLE      1
#define MPI_INT         2
#define MPI_MIN         1
#define MPI_MAX         2
#define MPI_SUM         3
#define MPI_IN_PLACE        ((void*)1)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_STATUS_IGNORE   ((MPI_Status*)0)

int MPI_Init(int* argc, char*** argv);
int MPI_Initialized(int* flag);
int MPI_Finalize(void);
int MPI_Finalized(int* flag);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Dims_create(int nnodes, int ndims, int dims[]);
int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[],
                    int reorder, MPI_Comm* cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int* source, int* dest);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
               void* recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request* req);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status statuses[]);

int sifv_mpi_shim_run(int nranks, void (*fn)(void* user, int rank), void* user);

#ifdef __cplusplus
}
#endif

#endif /* SIFV_MPI_SHIM_H */
