/*
 * Single-rank stand-in for the MPI API, used only to compile the reference
 * tycho2 sources (src/*.cc) into the CPU checker under oracle/_ref.
 *
 * Test infrastructure: nothing in the product links this file.
 *
 * Every communicator has exactly one rank (rank 0).  Collectives copy their
 * send buffer to the receive buffer.  Point-to-point calls can never be
 * reached with one partition (the reference only talks to adjacent ranks,
 * of which a one-partition mesh has none), so they fail loudly if called.
 * MPI-IO maps onto stdio, which is all that a single writer/reader needs.
 *
 * One rank's view of a multi-partition run: TYCHO_SHIM_RANK and
 * TYCHO_SHIM_SIZE (default 0 and 1) set what MPI_Comm_rank / MPI_Comm_size
 * report, so that the reference reads that rank's partition of a .pmesh.
 * With a size above 1, the only point-to-point exchange that a dump without
 * inter-rank sweeps reaches -- TychoMesh's constructor asking each
 * neighbouring rank for its cell and face across a partition side
 * (src/TychoMeshIO.cc:298-333) -- completes without a peer: sends are
 * dropped and receives read zeros, so getAdjCellFromSide /
 * getAdjFaceFromSide hold zeros.  A dump run that way must not read them;
 * probes and message counts still fail loudly.
 */
#ifndef TYCHO_ORACLE_MPI_SHIM_H
#define TYCHO_ORACLE_MPI_SHIM_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef FILE *MPI_File;
typedef struct { int count_bytes; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_SEEK_SET SEEK_SET

#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_DOUBLE 3
#define MPI_UINT64_T 4
#define MPI_INT 5

#define MPI_SUM 1
#define MPI_MAX 2

#define MPI_MODE_RDONLY 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_CREATE 4
#define MPI_MODE_EXCL 8

static inline size_t tycho_shim_type_size(MPI_Datatype t)
{
    switch (t) {
        case MPI_BYTE: case MPI_CHAR: return 1;
        case MPI_DOUBLE: case MPI_UINT64_T: return 8;
        case MPI_INT: return 4;
        default: return 0;
    }
}

static inline int tycho_shim_env(const char *name, int dflt)
{
    const char *v = getenv(name);
    return v ? atoi(v) : dflt;
}

static inline int tycho_shim_unreachable(const char *what)
{
    fprintf(stderr, "mpi shim: %s called with one rank\n", what);
    abort();
    return MPI_ERR_OTHER;
}

static inline int MPI_Init(int *argc, char ***argv)
{ (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Init_thread(int *argc, char ***argv, int req, int *prov)
{ (void)argc; (void)argv; *prov = req; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r)
{ (void)c; *r = tycho_shim_env("TYCHO_SHIM_RANK", 0); return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *s)
{ (void)c; *s = tycho_shim_env("TYCHO_SHIM_SIZE", 1); return MPI_SUCCESS; }
static inline int tycho_shim_view(void) { return tycho_shim_env("TYCHO_SHIM_SIZE", 1) > 1; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }

static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t,
                                MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    memmove(r, s, (size_t)n * tycho_shim_type_size(t));
    return MPI_SUCCESS;
}

static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return tycho_shim_unreachable("MPI_Send"); }
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *rq)
{
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c;
    if (!tycho_shim_view()) return tycho_shim_unreachable("MPI_Isend");
    *rq = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st)
{
    (void)s; (void)tag; (void)c; (void)st;
    if (!tycho_shim_view()) return tycho_shim_unreachable("MPI_Recv");
    memset(b, 0, (size_t)n * tycho_shim_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *rq)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)rq; return tycho_shim_unreachable("MPI_Irecv"); }
static inline int MPI_Iprobe(int s, int tag, MPI_Comm c, int *flag, MPI_Status *st)
{ (void)s; (void)tag; (void)c; (void)st; *flag = 0; return tycho_shim_unreachable("MPI_Iprobe"); }
static inline int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *n)
{ (void)st; (void)t; *n = 0; return tycho_shim_unreachable("MPI_Get_count"); }

static inline int MPI_Waitall(int n, MPI_Request *rq, MPI_Status *st)
{
    (void)rq; (void)st;
    return n == 0 || tycho_shim_view() ? MPI_SUCCESS : tycho_shim_unreachable("MPI_Waitall");
}
static inline int MPI_Waitany(int n, MPI_Request *rq, int *idx, MPI_Status *st)
{
    (void)rq; (void)st; (void)idx;
    return n == 0 ? MPI_SUCCESS : tycho_shim_unreachable("MPI_Waitany");
}

static inline int MPI_File_open(MPI_Comm c, const char *name, int mode, MPI_Info info, MPI_File *f)
{
    (void)c; (void)info;
    if (mode & MPI_MODE_RDONLY) {
        *f = fopen(name, "rb");
        return *f ? MPI_SUCCESS : MPI_ERR_OTHER;
    }
    if (mode & MPI_MODE_EXCL) {
        FILE *probe = fopen(name, "rb");
        if (probe) { fclose(probe); return MPI_ERR_OTHER; }
    }
    *f = fopen(name, "wb");
    return *f ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_File_delete(const char *name, MPI_Info info)
{ (void)info; return remove(name) == 0 ? MPI_SUCCESS : MPI_ERR_OTHER; }
static inline int MPI_File_close(MPI_File *f)
{ int r = fclose(*f); *f = NULL; return r == 0 ? MPI_SUCCESS : MPI_ERR_OTHER; }
static inline int MPI_File_seek(MPI_File f, MPI_Offset off, int whence)
{ return fseek(f, (long)off, whence) == 0 ? MPI_SUCCESS : MPI_ERR_OTHER; }
static inline int MPI_File_read(MPI_File f, void *b, int n, MPI_Datatype t, MPI_Status *st)
{
    (void)st;
    size_t bytes = (size_t)n * tycho_shim_type_size(t);
    return fread(b, 1, bytes, f) == bytes ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_File_write_at(MPI_File f, MPI_Offset off, const void *b, int n,
                                    MPI_Datatype t, MPI_Status *st)
{
    (void)st;
    size_t bytes = (size_t)n * tycho_shim_type_size(t);
    if (fseek(f, (long)off, SEEK_SET) != 0) return MPI_ERR_OTHER;
    return fwrite(b, 1, bytes, f) == bytes ? MPI_SUCCESS : MPI_ERR_OTHER;
}

#endif
