/* Test-infrastructure shim: a single-rank MPI so the reference CPU FMM, which
 * hard-defines FMM_MPI, runs as one process.  Collectives copy the local part;
 * broadcasts and barriers do nothing.  A datatype is its size in bytes. */
#pragma once
#include <cstring>
#include <memory>
#include <vector>
#include <fstream>

typedef int MPI_Comm;
typedef int MPI_Datatype;
#define MPI_COMM_WORLD 0
#define MPI_BYTE 1
#define MPI_DOUBLE 8
#define MPI_COMPLEX16 16
#define MPI_SUCCESS 0

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* out) { *out = count * old; return MPI_SUCCESS; }
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Allgatherv(const void* send, int sendcount, MPI_Datatype st, void* recv,
                          const int*, const int* displs, MPI_Datatype rt, MPI_Comm)
{
	if (send != recv)
		std::memmove((char*)recv + (size_t)displs[0] * rt, send, (size_t)sendcount * st);
	return MPI_SUCCESS;
}
inline int MPI_Alltoallv(const void* send, const int* sendcounts, const int* sdispls, MPI_Datatype st,
                         void* recv, const int*, const int* rdispls, MPI_Datatype rt, MPI_Comm)
{
	std::memmove((char*)recv + (size_t)rdispls[0] * rt, (const char*)send + (size_t)sdispls[0] * st,
	             (size_t)sendcounts[0] * st);
	return MPI_SUCCESS;
}
