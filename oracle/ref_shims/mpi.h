// Plumbing shim: the oracle is one process, so MPI is a single-rank stand-in.
// Communicators, requests and infos are inert handles; a datatype handle
// carries its element size; rank 0 of 1, and a reduction or gather over the
// one rank copies its input to its output.
#pragma once
#include <cstring>
typedef void* MPI_Comm;
typedef void* MPI_Request;
typedef void* MPI_Info;
typedef void* MPI_Datatype;
typedef int MPI_Op;
typedef long MPI_Offset;
#define MPI_SUCCESS 0
#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_INFO_NULL ((MPI_Info)0)
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_DOUBLE ((MPI_Datatype)(long)sizeof(double))
#define MPI_FLOAT ((MPI_Datatype)(long)sizeof(float))
#define MPI_LONG_LONG ((MPI_Datatype)(long)sizeof(long long))

inline int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}

inline int MPI_Comm_size(MPI_Comm, int* size) {
    *size = 1;
    return MPI_SUCCESS;
}

inline int MPI_Comm_split(MPI_Comm comm, int, int, MPI_Comm* out) {
    *out = comm;
    return MPI_SUCCESS;
}

inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, int,
    MPI_Comm) {
    if (send != recv) {
        std::memmove(recv, send, size_t(count) * size_t((long)type));
    }
    return MPI_SUCCESS;
}

inline int MPI_Allgather(const void* send, int count, MPI_Datatype type, void* recv, int,
    MPI_Datatype, MPI_Comm) {
    if (send != recv) {
        std::memmove(recv, send, size_t(count) * size_t((long)type));
    }
    return MPI_SUCCESS;
}
