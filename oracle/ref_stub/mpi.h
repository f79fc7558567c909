/* Single-rank stand-in for <mpi.h>, used only to compile the reference
 * CapacMD sources as a CPU oracle (test infrastructure, never shipped).
 *
 * With one rank every MPI loop in the reference runs `an_id = 1 .. np-1`
 * zero times (force.c:438, force.c:2264, bicg_stab.c:150, bicg_stab.c:209),
 * so point-to-point calls are never reached; they abort if they ever are.
 * MPI_Bcast with a single rank is the identity.
 */
#ifndef CAPAC_ORACLE_MPI_STUB_H
#define CAPAC_ORACLE_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_ANY_SOURCE (-1)

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return 0; }
static inline int MPI_Bcast(void *buf, int n, MPI_Datatype t, int root, MPI_Comm c)
{
    (void)buf; (void)n; (void)t; (void)root; (void)c;
    return 0;
}
static inline int MPI_Send(const void *buf, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
    (void)buf; (void)n; (void)t; (void)dest; (void)tag; (void)c;
    fprintf(stderr, "oracle mpi stub: MPI_Send reached with one rank\n");
    abort();
}
static inline int MPI_Recv(void *buf, int n, MPI_Datatype t, int src, int tag, MPI_Comm c,
                           MPI_Status *st)
{
    (void)buf; (void)n; (void)t; (void)src; (void)tag; (void)c; (void)st;
    fprintf(stderr, "oracle mpi stub: MPI_Recv reached with one rank\n");
    abort();
}

#endif
