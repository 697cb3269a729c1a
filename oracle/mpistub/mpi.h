/*
 * Single-rank MPI stand-in used ONLY to compile the reference library
 * (fvhyper/src/*.cpp) into the oracle under oracle/_ref/.  Test
 * infrastructure: nothing in the product links this file.
 *
 * With one rank every MPI call site in the reference is either skipped
 * (guarded by `pool.size > 1`, fvhyper/src/explicit.cpp:639-648,730,733,746)
 * or loops over zero peers (fvhyper/src/mesh.cpp:679-798 with no ghost
 * elements), so every function here is a no-op that reports success.
 */
#ifndef FVREF_MPI_STUB_H
#define FVREF_MPI_STUB_H

#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_UNSIGNED 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return MPI_SUCCESS; }
inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Request_free(MPI_Request*) { return MPI_SUCCESS; }

#endif
