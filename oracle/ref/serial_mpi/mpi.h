/* Single-process stand-in for the handful of MPI entry points the BabelSim
 * sources reference.  Test infrastructure only: it lets the reference's own
 * finite-volume sources compile and run serially as the oracle, where no MPI
 * implementation is installed.  Every collective degenerates to a copy on a
 * one-rank communicator; point-to-point and neighbourhood calls are never
 * reached serially (the reference returns early when !distributed()) and
 * report an error if they ever are. */
#ifndef BABELSIM_ORACLE_SERIAL_MPI_H
#define BABELSIM_ORACLE_SERIAL_MPI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MAX_ERROR_STRING 256
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_UNWEIGHTED ((int*)0)
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline size_t bsoracle_type_size(MPI_Datatype t) {
    return t == MPI_CHAR ? 1u : t == MPI_INT ? sizeof(int) : t == MPI_DOUBLE ? sizeof(double) : 0u;
}
static inline int bsoracle_state(int query, int set) {
    static int initialized = 0, finalized = 0;
    if (set == 1) initialized = 1;
    if (set == 2) finalized = 1;
    return query == 1 ? initialized : finalized;
}
static inline int bsoracle_unreachable(const char* name) {
    fprintf(stderr, "serial MPI stand-in: %s is not available in a one-rank run\n", name);
    return MPI_ERR_OTHER;
}
static inline int MPI_Init(int*, char***) { bsoracle_state(0, 1); return MPI_SUCCESS; }
static inline int MPI_Init_thread(int*, char***, int, int* provided) {
    bsoracle_state(0, 1); if (provided) *provided = 0; return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { bsoracle_state(0, 2); return MPI_SUCCESS; }
static inline int MPI_Initialized(int* flag) { *flag = bsoracle_state(1, 0); return MPI_SUCCESS; }
static inline int MPI_Finalized(int* flag) { *flag = bsoracle_state(2, 0); return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); }
static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm* comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Error_string(int code, char* text, int* length) {
    *length = snprintf(text, MPI_MAX_ERROR_STRING, "serial MPI error %d", code);
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* in, void* out, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (in != out) memmove(out, in, (size_t)count * bsoracle_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* in, int count, MPI_Datatype t, void* out, int, MPI_Datatype, MPI_Comm) {
    if (in != out) memmove(out, in, (size_t)count * bsoracle_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Alltoall(const void* in, int count, MPI_Datatype t, void* out, int, MPI_Datatype, MPI_Comm) {
    if (in != out) memmove(out, in, (size_t)count * bsoracle_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Alltoallv(const void* in, const int* counts, const int* displs, MPI_Datatype t,
                                void* out, const int*, const int* rdispls, MPI_Datatype, MPI_Comm) {
    const size_t s = bsoracle_type_size(t);
    memmove((char*)out + (size_t)rdispls[0] * s, (const char*)in + (size_t)displs[0] * s, (size_t)counts[0] * s);
    return MPI_SUCCESS;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
    return bsoracle_unreachable("MPI_Send");
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
    return bsoracle_unreachable("MPI_Recv");
}
static inline int MPI_Dist_graph_create_adjacent(MPI_Comm, int, const int*, const int*, int, const int*,
                                                 const int*, MPI_Info, int, MPI_Comm*) {
    return bsoracle_unreachable("MPI_Dist_graph_create_adjacent");
}
static inline int MPI_Ineighbor_alltoallv(const void*, const int*, const int*, MPI_Datatype, void*, const int*,
                                          const int*, MPI_Datatype, MPI_Comm, MPI_Request*) {
    return bsoracle_unreachable("MPI_Ineighbor_alltoallv");
}
static inline int MPI_Ialltoallv(const void*, const int*, const int*, MPI_Datatype, void*, const int*,
                                 const int*, MPI_Datatype, MPI_Comm, MPI_Request*) {
    return bsoracle_unreachable("MPI_Ialltoallv");
}
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }

#endif
