/* Test infrastructure only: a single-rank stand-in for the MPI calls the ExaCA reference makes, so
 * that its unmodified sources compile here (no MPI is installed). World size is 1 and rank 0.
 * Reductions, gathers and all-reduces copy the local value; broadcasts and barriers do nothing;
 * point-to-point calls only ever address MPI_PROC_NULL at one rank and are no-ops; MPI_Waitany
 * reports MPI_UNDEFINED (no pending receives). MPI_Wtime is a steady clock in seconds.
 * Nothing in the product includes this file. */
#ifndef EXACA_ORACLE_MPI_SHIM_H
#define EXACA_ORACLE_MPI_SHIM_H

#include <chrono>
#include <cstring>
#include <stdexcept>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_UNDEFINED (-32766)
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_UNSIGNED_LONG 4
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

inline size_t exaca_shim_type_size(MPI_Datatype t) {
    switch (t) {
    case MPI_INT: return sizeof(int);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_UNSIGNED_LONG: return sizeof(unsigned long);
    default: throw std::runtime_error("mpi shim: unknown datatype");
    }
}

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_size(MPI_Comm, int *np) {
    *np = 1;
    return 0;
}
inline int MPI_Comm_rank(MPI_Comm, int *id) {
    *id = 0;
    return 0;
}
inline double MPI_Wtime() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    std::memcpy(r, s, n * exaca_shim_type_size(t));
    return 0;
}
inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    std::memcpy(r, s, n * exaca_shim_type_size(t));
    return 0;
}
inline int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm) {
    std::memcpy(r, s, n * exaca_shim_type_size(t));
    return 0;
}
inline void exaca_shim_require_null(int peer) {
    if (peer != MPI_PROC_NULL)
        throw std::runtime_error("mpi shim: point-to-point with a real peer at world size 1");
}
inline int MPI_Send(const void *, int, MPI_Datatype, int peer, int, MPI_Comm) {
    exaca_shim_require_null(peer);
    return 0;
}
inline int MPI_Recv(void *, int, MPI_Datatype, int peer, int, MPI_Comm, MPI_Status *) {
    exaca_shim_require_null(peer);
    return 0;
}
inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int p1, int, void *, int, MPI_Datatype, int p2, int,
                        MPI_Comm, MPI_Status *) {
    exaca_shim_require_null(p1);
    exaca_shim_require_null(p2);
    return 0;
}
inline int MPI_Isend(const void *, int, MPI_Datatype, int peer, int, MPI_Comm, MPI_Request *req) {
    exaca_shim_require_null(peer);
    *req = MPI_REQUEST_NULL;
    return 0;
}
inline int MPI_Irecv(void *, int, MPI_Datatype, int peer, int, MPI_Comm, MPI_Request *req) {
    exaca_shim_require_null(peer);
    *req = MPI_REQUEST_NULL;
    return 0;
}
inline int MPI_Waitany(int, MPI_Request *, int *idx, MPI_Status *) {
    *idx = MPI_UNDEFINED;
    return 0;
}
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }

#endif
