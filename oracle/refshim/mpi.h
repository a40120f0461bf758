// TEST INFRASTRUCTURE ONLY -- used to compile the reference's own sources into
// oracle/_ref/ (the checker); nothing in the product includes it.
//
// Single-rank stand-in for the subset of the MPI C interface that the
// reference calls (src/core/mpi/Communicator.hpp:17-260,
// src/MPIindex/MPIindex.hpp, src/Simulation/Simulation.cpp:816,
// src/Operator/BlockMatrix_definitions.hpp:355-400).  With one rank every
// collective is a copy, every barrier is a no-op and a message to oneself is
// delivered through a per-process mailbox.
#pragma once
#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; };

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_SUCCESS 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_REQUEST_NULL 0

// datatype handles carry their size in bytes in the low byte
#define MPI_CHAR            ((MPI_Datatype)(0x100 | 1))
#define MPI_UNSIGNED_CHAR   ((MPI_Datatype)(0x200 | 1))
#define MPI_C_BOOL          ((MPI_Datatype)(0x300 | 1))
#define MPI_SHORT           ((MPI_Datatype)(0x400 | 2))
#define MPI_INT             ((MPI_Datatype)(0x500 | 4))
#define MPI_UINT32_T        ((MPI_Datatype)(0x600 | 4))
#define MPI_FLOAT           ((MPI_Datatype)(0x700 | 4))
#define MPI_UNSIGNED_LONG   ((MPI_Datatype)(0x800 | 8))
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)(0x900 | 8))
#define MPI_DOUBLE          ((MPI_Datatype)(0xa00 | 8))
#define MPI_C_FLOAT_COMPLEX ((MPI_Datatype)(0xb00 | 8))
#define MPI_LONG_DOUBLE     ((MPI_Datatype)(0xc00 | 16))
#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)(0xd00 | 16))

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)

extern "C" {
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided);
int MPI_Query_thread(int* provided);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm comm);
double MPI_Wtime(void);
}
