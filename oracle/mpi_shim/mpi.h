/*
 * Thread-rank MPI stand-in — TEST INFRASTRUCTURE ONLY.
 *
 * This header lets the reference's CPU solver library (PaScaLTDMA in
 * libs/pascal_tdma/cpu/pascal_tdma.cpp and FilteredTDMA in
 * libs/filtered_tdma/cpu/filtered_tdma.cpp) compile unmodified on a machine
 * without MPI.  Ranks are threads of one process; a communicator is a shared
 * object that the rank threads rendezvous on.  Only the calls those two files
 * make are provided:
 *   MPI_Allgather (MPI_INT), MPI_Type_create_subarray (2-D, C order, doubles),
 *   MPI_Type_commit/free, MPI_Ialltoallw, MPI_Isend/Irecv, MPI_Wait/Waitall,
 *   MPI_Barrier, MPI_Wtime.
 * Non-blocking collectives complete inside the call (every rank issues them
 * in the same order, so this cannot deadlock); point-to-point messages are
 * matched by (source, destination, tag) at wait time.
 *
 * The reference's channel-flow GPU sources (apps/channel_gpu/
 * MomentumSolverGPU.cu, PressureSolverGPU.cu) are also compiled against this
 * header, for their coefficient-build kernels only (oracle/_ref/
 * libref_channel.so).  The further calls those files name -- MPI_Allreduce,
 * MPI_Alltoall, MPI_Alltoallv, MPI_Bcast -- are declared so that they compile
 * and throw if ever called: nothing that drives those kernels calls them.
 *
 * The product library never includes this file.  It is used by oracle/_ref
 * (the reference built from its own sources) and the CPU baseline only.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct shim_comm* MPI_Comm;
typedef struct shim_type* MPI_Datatype;
typedef struct shim_req*  MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

extern struct shim_type shim_type_double;
extern struct shim_type shim_type_int;

#define MPI_DOUBLE (&shim_type_double)
#define MPI_INT (&shim_type_int)
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)
#define MPI_PROC_NULL (-2)
#define MPI_ORDER_C 56
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_COMM_NULL ((MPI_Comm)0)

typedef int MPI_Op;
#define MPI_MAX 1
#define MPI_SUM 2

int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                  void* recvbuf, int recvcount, MPI_Datatype recvtype,
                  MPI_Comm comm);
int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order, MPI_Datatype oldtype,
                             MPI_Datatype* newtype);
int MPI_Type_commit(MPI_Datatype* type);
int MPI_Type_free(MPI_Datatype* type);
int MPI_Ialltoallw(const void* sendbuf, const int sendcounts[], const int sdispls[],
                   const MPI_Datatype sendtypes[], void* recvbuf,
                   const int recvcounts[], const int rdispls[],
                   const MPI_Datatype recvtypes[], MPI_Comm comm,
                   MPI_Request* request);
int MPI_Isend(const void* buf, int count, MPI_Datatype datatype, int dest,
              int tag, MPI_Comm comm, MPI_Request* request);
int MPI_Irecv(void* buf, int count, MPI_Datatype datatype, int source,
              int tag, MPI_Comm comm, MPI_Request* request);
int MPI_Wait(MPI_Request* request, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request requests[], MPI_Status statuses[]);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);

/* Declared for the channel sources; they throw (see above). */
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype,
                  MPI_Op op, MPI_Comm comm);
int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                 int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Alltoallv(const void* sendbuf, const int sendcounts[], const int sdispls[],
                  MPI_Datatype sendtype, void* recvbuf, const int recvcounts[],
                  const int rdispls[], MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Bcast(void* buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm);

/* Shim control (not MPI): create a communicator of `size` thread ranks and
 * bind the calling thread to `rank` of it. */
MPI_Comm shim_comm_create(int size);
void shim_comm_destroy(MPI_Comm comm);
void shim_bind_rank(MPI_Comm comm, int rank);

#ifdef __cplusplus
}
#endif

#endif
