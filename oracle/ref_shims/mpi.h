// Plumbing shim: the oracle is single-process, so MPI handles are inert types.
#pragma once
typedef void* MPI_Comm;
typedef void* MPI_Request;
typedef void* MPI_Info;
typedef void* MPI_Datatype;
typedef long MPI_Offset;
