/* Single-rank stand-in for the eleven MPI symbols VMaChine calls.
 *
 * Test infrastructure only: it lets the reference C++ sources compile and run
 * as one rank (one walker) in a container without an MPI installation.  Every
 * collective degenerates to a copy (Reduce) or a no-op (Bcast, Barrier), which
 * is exactly what MPI does with a communicator of size one.  MPI_Bcast is a
 * no-op on purpose: the reference broadcasts an `int` declared as MPI_DOUBLE
 * (src/system.cpp:130), and copying 8 bytes there would overrun it.
 */
#pragma once
#include <cstdlib>
#include <cstring>
#include <ctime>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 0

static inline int vmcstub_type_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }

static inline int MPI_Initialized(int *flag) { *flag = 1; return 0; }
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op,
                             int, MPI_Comm)
{
    if (send != recv) std::memcpy(recv, send, size_t(count) * size_t(vmcstub_type_size(t)));
    return 0;
}
static inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
static inline double MPI_Wtime()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return double(ts.tv_sec) + 1e-9 * double(ts.tv_nsec);
}
