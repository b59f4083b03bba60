/*
 * mpi.h -- a one-rank stand-in for the MPI calls the wloop modules make.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref).  Every module guards its
 * communication with NPROC > 1; what remains unguarded (broadcasts and
 * reductions over the one rank, lnkplaq.c, wloop.c) becomes a copy.  A
 * point-to-point call cannot happen with one rank and aborts if reached.
 */
#ifndef WLREF_MPI_H
#define WLREF_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_SUCCESS 0

int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op, int root,
               MPI_Comm comm);
int MPI_Allreduce(void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Send(void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm,
             MPI_Status *status);
double MPI_Wtime(void);

#endif
