/*
 * Single-rank stand-in for the MPI API, used only to compile the reference's
 * CPU path as a test oracle (test infrastructure; never linked into the
 * product library).
 *
 * The reference calls MPI for a 3-D Cartesian decomposition
 * (src/init_MPI.cpp:24-60), halo exchange (src/MPI_send_recv*.cpp) and a few
 * reductions (src/calc_CFL.cpp:303-313).  With one rank every neighbour is
 * MPI_PROC_NULL, so a Sendrecv moves nothing, a reduction is a copy and a
 * barrier is a no-op.  MPI_PROC_NULL is negative because the reference skips
 * packing when a neighbour rank is < 0 (src/MPI_send_recv_FLOAT.cpp:424).
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_CHAR 1
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
#define MPI_INT 40
#define MPI_MIN 100
#define MPI_MAX 101
#define MPI_SUM 102
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_SUCCESS 0

static inline int oracle_mpi_type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_CHAR: return 1;
    case MPI_FLOAT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_INT: return 4;
    default: return 1;
    }
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_free(MPI_Comm *) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code)
{
    fprintf(stderr, "MPI_Abort(%d)\n", code);
    fflush(stdout);
    exit(code & 0xff ? code & 0xff : 1);
}
static inline int MPI_Get_processor_name(char *name, int *len)
{
    strcpy(name, "oracle");
    *len = 6;
    return 0;
}
static inline int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *c)
{
    *c = 0;
    return 0;
}
static inline int MPI_Cart_shift(MPI_Comm, int, int, int *src, int *dst)
{
    *src = MPI_PROC_NULL;
    *dst = MPI_PROC_NULL;
    return 0;
}
static inline int MPI_Cart_coords(MPI_Comm, int, int n, int *coords)
{
    for (int i = 0; i < n; i++) coords[i] = 0;
    return 0;
}
static inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int,
                               void *, int, MPI_Datatype, int, int,
                               MPI_Comm, MPI_Status *)
{
    return 0; /* both partners are MPI_PROC_NULL with one rank */
}
static inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    memcpy(out, in, (size_t)n * oracle_mpi_type_size(t));
    return 0;
}

#endif
