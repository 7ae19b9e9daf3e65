/* Single-process stand-in for the subset of MPI that the reference driver
 * (src/GeneralModel/antelope.cpp) calls, so the unmodified reference sources
 * compile without an MPI installation.  Test infrastructure only: this header
 * is on the include path of the oracle/_ref build and nowhere else.
 *
 * Semantics:
 *  - MPI_Comm_rank / MPI_Comm_size return REF_RANK / REF_SIZE from the
 *    environment (defaults 0 / 1).  With REF_SIZE > 1 each process computes the
 *    k-slice that ParaRange (utility.h:104-115) assigns to that rank, which is
 *    how the timed CPU baseline spreads the reference over host cores.
 *  - Reductions and gathers are no-ops: in the reference every one of them is
 *    either in place on the master (antelope.cpp:366,435,487,496,506) or feeds
 *    only stdout, so a single rank already holds the full result.
 *  - With REF_DUMP set to a path prefix, every MPI_Reduce also writes the
 *    calling rank's buffer (the receive buffer for MPI_IN_PLACE) as raw bytes
 *    to <prefix>.<call number>.bin, call numbers counting from 0 in call
 *    order.  At the final reduce (antelope.cpp:482-512) these are the rank's
 *    partial k-sums -- inter and intra current per axis (Nt complex each, in
 *    the order x inter, x intra, y inter, ...), then the weighted density
 *    matrix (Nt x N^2 complex) -- so the k-slice that ParaRange gives one
 *    emulated rank can be compared with another implementation's slice, and
 *    the slices of all ranks summed in rank order give the whole grid.
 */
#ifndef ORACLE_REFSHIM_MPI_H
#define ORACLE_REFSHIM_MPI_H

#include <stdio.h>
#include <stdlib.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef void MPI_User_function(void *, void *, int *, MPI_Datatype *);

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_DOUBLE 1
#define MPI_DOUBLE_COMPLEX 2
#define MPI_IN_PLACE ((void *)1)

static inline int refshim_env_int(const char *name, int dflt)
{
    const char *v = getenv(name);
    return v ? atoi(v) : dflt;
}

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank)
{
    *rank = refshim_env_int("REF_RANK", 0);
    return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm, int *size)
{
    *size = refshim_env_int("REF_SIZE", 1);
    return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Op_create(MPI_User_function *, int, MPI_Op *op)
{
    *op = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm)
{
    static int calls = 0;
    const char *prefix = getenv("REF_DUMP");
    const int call = calls++;
    if (!prefix) return MPI_SUCCESS;
    const void *buf = send == MPI_IN_PLACE ? recv : send;
    const size_t elem = type == MPI_DOUBLE_COMPLEX ? 16 : 8;
    char path[4096];
    snprintf(path, sizeof(path), "%s.%d.bin", prefix, call);
    FILE *f = fopen(path, "wb");
    if (!f || fwrite(buf, elem, (size_t)count, f) != (size_t)count) {
        fprintf(stderr, "refshim: cannot write %s\n", path);
        exit(EXIT_FAILURE);
    }
    fclose(f);
    return MPI_SUCCESS;
}
static inline int MPI_Gatherv(const void *, int, MPI_Datatype, void *, const int *, const int *,
                              MPI_Datatype, int, MPI_Comm)
{
    return MPI_SUCCESS;
}

#endif
