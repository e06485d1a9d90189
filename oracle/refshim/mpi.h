/*
 * Single-rank stand-in for the MPI calls made by the reference's CPU path.
 *
 * TEST INFRASTRUCTURE ONLY: this header exists so that the reference sources
 * (weno/src/update.cpp, FlowField.cpp, ParticleTrack.cpp) can be compiled
 * unmodified into the oracle binary under oracle/_ref.  It is never linked
 * into the product library.
 *
 * Semantics: one process owns the whole periodic block.  A Cartesian shift
 * therefore names the process itself, MPI_Sendrecv is a copy of the send
 * buffer into the receive buffer (which turns the reference's HaloTransfer,
 * weno/src/update.cpp:894-1054, into a periodic wrap), and every reduction of
 * one contribution is a copy.  A datatype handle is its size in bytes.
 */
#ifndef GKS_REFSHIM_MPI_H
#define GKS_REFSHIM_MPI_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_DOUBLE_PRECISION ((MPI_Datatype)sizeof(double))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_SUM ((MPI_Op)0)
#define MPI_MAX ((MPI_Op)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

static inline int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *c)
{
    *c = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_coords(MPI_Comm, int, int nd, int *coords)
{
    for (int i = 0; i < nd; ++i) coords[i] = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_shift(MPI_Comm, int, int, int *src, int *dst)
{
    *src = 0;
    *dst = 0;
    return MPI_SUCCESS;
}

static inline int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int, int,
                               void *rbuf, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *)
{
    memcpy(rbuf, sbuf, (size_t)scount * (size_t)stype);
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void *sbuf, void *rbuf, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    memcpy(rbuf, sbuf, (size_t)n * (size_t)t);
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *sbuf, void *rbuf, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    memcpy(rbuf, sbuf, (size_t)n * (size_t)t);
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

/* Present only in commented-out code of the reference; declared for completeness. */
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_SUCCESS; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_SUCCESS; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return MPI_SUCCESS; }

#endif
