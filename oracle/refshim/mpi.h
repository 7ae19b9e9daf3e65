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
 */
#ifndef ORACLE_REFSHIM_MPI_H
#define ORACLE_REFSHIM_MPI_H

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
static inline int MPI_Reduce(const void *, void *, int, MPI_Datatype, MPI_Op, int, MPI_Comm)
{
    return MPI_SUCCESS;
}
static inline int MPI_Gatherv(const void *, int, MPI_Datatype, void *, const int *, const int *,
                              MPI_Datatype, int, MPI_Comm)
{
    return MPI_SUCCESS;
}

#endif
