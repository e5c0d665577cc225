/*
 * Single-rank MPI stand-in used ONLY to compile the reference DSMC solver
 * (andeplane/master code/base_code/program/dsmc/) as a CPU oracle and CPU
 * baseline.  Test infrastructure: nothing in the shipped library includes it.
 *
 * With one rank every collective the reference issues reduces to a copy:
 *   MPI_Reduce  (dsmc/statisticssampler.cpp:56-57, dsmc/system.cpp:103,337,
 *                dsmc/statisticalproperty.cpp:34,95,287-288,...) -> memcpy
 *   MPI_Send/Recv (dsmc/system.cpp:80-90) are only reached when the
 *                 topology has more than one processor; they abort here.
 *   MPI_Wtime   -> CLOCK_MONOTONIC seconds.
 */
#pragma once
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <ctime>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_ANY_SOURCE (-1)
#define MPI_SUM 0
#define MPI_INT 1
#define MPI_LONG 2
#define MPI_UNSIGNED_LONG 3
#define MPI_DOUBLE 4

static inline size_t mpi_stub_type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_INT: return sizeof(int);
        case MPI_LONG: return sizeof(long);
        case MPI_UNSIGNED_LONG: return sizeof(unsigned long);
        case MPI_DOUBLE: return sizeof(double);
    }
    return 0;
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline double MPI_Wtime() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    std::memcpy(recv, send, count * mpi_stub_type_size(t));
    return 0;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) {
    std::fprintf(stderr, "mpi stub: MPI_Send needs more than one rank\n");
    std::abort();
}
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
    std::fprintf(stderr, "mpi stub: MPI_Recv needs more than one rank\n");
    std::abort();
}
