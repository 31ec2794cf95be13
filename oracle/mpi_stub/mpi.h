/*
 * mpi.h -- a single-process stand-in for the subset of MPI that the
 * reference's multi-GPU library uses (ResistiveMHD_multiGPU_cuda/
 * ResistiveMHD2D_GPU/mpi.hpp:1-40 includes <mpi.h>; mpi.cu and
 * resistiveMHD2D.cu call the functions below).  TEST INFRASTRUCTURE ONLY:
 * oracle/build_ref.py puts this directory first on the include path when it
 * builds that library unmodified for the host, as a checker of this
 * project's CT-Contact EMF and wall restatements.
 *
 * World of one rank: rank 0 of 1, MPI_Dims_create gives a 1 x 1 grid, so
 * every neighbour is the rank itself.  MPI_Sendrecv with source == dest ==
 * self delivers the send buffer into the receive buffer (the message the
 * call sends is the one it receives, as MPI specifies for a self-exchange),
 * MPI_Allreduce copies (the reduction of one contribution), MPI_Barrier does
 * nothing.  A datatype is represented by its extent in bytes.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H

#include <stddef.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;   /* extent in bytes */
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_C_BOOL ((MPI_Datatype)sizeof(bool))
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_LOR 4

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank)
{
    *rank = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm, int *size)
{
    *size = 1;
    return MPI_SUCCESS;
}
/* Fills the zero entries of dims so that their product is nnodes (= 1). */
static inline int MPI_Dims_create(int, int ndims, int *dims)
{
    for (int d = 0; d < ndims; ++d)
        if (dims[d] == 0) dims[d] = 1;
    return MPI_SUCCESS;
}
/* The extent of a struct type: the end of its furthest block. */
static inline int MPI_Type_create_struct(int count, const int *lens, const MPI_Aint *offsets,
                                         const MPI_Datatype *types, MPI_Datatype *out)
{
    long ext = 0;
    for (int k = 0; k < count; ++k) {
        const long end = offsets[k] + (long)lens[k] * types[k];
        if (end > ext) ext = end;
    }
    *out = (MPI_Datatype)ext;
    return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int, int,
                               void *recvbuf, int recvcount, MPI_Datatype recvtype, int, int, MPI_Comm,
                               MPI_Status *status)
{
    size_t n = (size_t)sendcount * (size_t)sendtype;
    const size_t cap = (size_t)recvcount * (size_t)recvtype;
    if (n > cap) n = cap;
    if (n) memmove(recvbuf, sendbuf, n);
    if (status) {
        status->MPI_SOURCE = 0;
        status->MPI_TAG = 0;
        status->MPI_ERROR = MPI_SUCCESS;
    }
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op,
                                MPI_Comm)
{
    if (sendbuf != recvbuf) memmove(recvbuf, sendbuf, (size_t)count * (size_t)type);
    return MPI_SUCCESS;
}

#endif
