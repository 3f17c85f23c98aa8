/*
 * Stand-in for <mpi.h>, used ONLY to compile the reference's hot-path C
 * sources into the parity checker under oracle/_ref/.
 *
 * This is test infrastructure, not product code.  MPI_Comm_rank / _size
 * answer rank 0 of 1 (the reference reads its pid and world size from
 * latticeMesh.parallel on the path, not from MPI).  At world size 1 the
 * reference never posts a message (sendPdfField.c:10 returns early, the
 * sync* helpers loop over zero peers).  For multi-rank checks the harness
 * runs every rank of a partitioned mesh in one process, one thread per rank
 * (oracle/ref_harness.c, ref_ranks_*): MPI_Isend, MPI_Irecv and MPI_Waitall
 * then pass messages between the threads through an in-process mailbox
 * (oracle/mpi_stub/mpi_stub.c), matched by source rank and tag as MPI
 * matches them.  Every wait is bounded; a receive that is never matched
 * returns an error and is counted (mplb_stub_failures).
 */
#ifndef MPLB_ORACLE_MPI_STUB_H
#define MPLB_ORACLE_MPI_STUB_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef int MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_SUM 1
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_RDONLY 4
#define MPI_SEEK_SET 0

static inline size_t mplb_stub_size(MPI_Datatype t) {
    switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_FLOAT: return sizeof(float);
    default: return sizeof(double);
    }
}

static inline int MPI_Init(int* c, char*** v) { (void)c; (void)v; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
/* Point-to-point calls between the rank threads of one process
 * (mpi_stub.c).  A send is buffered: it completes at once. */
int MPI_Isend(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* r);
int MPI_Irecv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request* r);
int MPI_Waitall(int n, MPI_Request* r, MPI_Status* s);
/* The calling thread acts as rank `rank` (the sender of its messages). */
void mplb_stub_set_rank(int rank);
/* Receives that gave up waiting since the last reset; reset clears the
 * mailbox too. */
int mplb_stub_failures(void);
void mplb_stub_reset(void);
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return 0; }
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return 0; }
/* Sum over the rank threads (mpi_stub.c); with one rank, the contribution. */
int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
/* Number of rank threads taking part in MPI_Allreduce (1 outside ref_ranks_*). */
void mplb_stub_set_world(int world);

#endif
