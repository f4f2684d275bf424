/*
 * Single-rank MPI stand-in used ONLY to compile the reference's CPU kernels
 * (src/utils/utils.cpp, src/decomp/slab/reorder_slab*.cpp) into the test
 * oracle under oracle/_ref/.  Test infrastructure: nothing in the product
 * links it.
 *
 * utils.cpp needs MPI_Comm, MPI_Reduce, MPI_Comm_rank, MPI_Barrier,
 * MPI_DOUBLE, MPI_MAX and MPI_COMM_WORLD (utils.cpp:12-20).  With one rank a
 * reduction is a copy and a barrier is a no-op.
 */
#ifndef PM_ORACLE_MPI_SHIM_H
#define PM_ORACLE_MPI_SHIM_H
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_COMM_NULL ((MPI_Comm)-1)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_MAX ((MPI_Op)1)
#define MPI_SUCCESS 0

static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype dt,
                             MPI_Op, int, MPI_Comm) {
    memcpy(recv, send, (size_t)count * (size_t)dt);
    return MPI_SUCCESS;
}
#endif
