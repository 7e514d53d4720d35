/* ORACLE / TEST INFRASTRUCTURE — a one-process stand-in for the MPI API, so
 * that the reference's complete driver (its src/main.cpp with everything
 * else) builds and runs here with n_sr = 1 as the checker of qp_driver's
 * output files.  Only the calls and constants that driver uses exist; with a
 * single rank every reduction, broadcast and all-reduce is a copy (or
 * nothing), and the point-to-point calls, which the driver only makes
 * between two different ranks, end the process if they are ever reached.
 * Nothing here is MPI's code: it is the semantics of one rank written out. */
#ifndef QUILL_ORACLE_MPI_STUB_H
#define QUILL_ORACLE_MPI_STUB_H

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef size_t MPI_Datatype; /* the element size in bytes */
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
    int count_bytes_;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

#define MPI_CHAR ((MPI_Datatype)sizeof(char))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_LONG ((MPI_Datatype)sizeof(long))
#define MPI_UNSIGNED_LONG ((MPI_Datatype)sizeof(unsigned long))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_CXX_BOOL ((MPI_Datatype)sizeof(bool))

#define MPI_SUM 1
#define MPI_MAX 2

static inline void mpi_stub_unreachable_(const char* what) {
    fprintf(stderr, "mpi stub: %s needs a second rank (one-process build)\n", what);
    exit(3);
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); return code; }
static inline int MPI_Get_processor_name(char* name, int* len) {
    strcpy(name, "localhost");
    *len = (int)strlen(name);
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
/* one rank: the result is the rank's own contribution */
static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    if (send != MPI_IN_PLACE && send != recv) memmove(recv, send, (size_t)count * t);
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    return MPI_Reduce(send, recv, count, t, op, 0, c);
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
    mpi_stub_unreachable_("MPI_Send");
    return 1;
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
    mpi_stub_unreachable_("MPI_Recv");
    return 1;
}
static inline int MPI_Probe(int, int, MPI_Comm, MPI_Status*) {
    mpi_stub_unreachable_("MPI_Probe");
    return 1;
}
static inline int MPI_Get_count(const MPI_Status*, MPI_Datatype, int*) {
    mpi_stub_unreachable_("MPI_Get_count");
    return 1;
}
static inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype, int, int, MPI_Comm,
                               MPI_Status*) {
    mpi_stub_unreachable_("MPI_Sendrecv");
    return 1;
}
static inline int MPI_Sendrecv_replace(void*, int, MPI_Datatype, int, int, int, int, MPI_Comm, MPI_Status*) {
    mpi_stub_unreachable_("MPI_Sendrecv_replace");
    return 1;
}
/* derived types: only their extent is used (the exchange is never reached) */
static inline int MPI_Type_create_struct(int, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Datatype* t) {
    *t = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Type_create_resized(MPI_Datatype, MPI_Aint, MPI_Aint extent, MPI_Datatype* t) {
    *t = (MPI_Datatype)extent;
    return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }

#endif
