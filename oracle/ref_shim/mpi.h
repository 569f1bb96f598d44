/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference's own
 * hot-path headers on the CPU as a test oracle (oracle/_ref).  Every
 * communicator has exactly one rank, so reductions and broadcasts are copies
 * (or no-ops when in place), and a send/receive to "self" is a copy.
 *
 * This is test infrastructure; nothing in the product links it.
 */
#pragma once
#include <cstring>
#include <cstdint>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; };

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_SUCCESS 0
#define MPI_DATATYPE_NULL 0
#define MPI_BYTE 1
#define MPI_INT 4
#define MPI_FLOAT 5
#define MPI_DOUBLE 8
#define MPI_INT64_T 9
#define MPI_UINT64_T 10
#define MPI_UINT 11
#define MPI_UINT32_T 11
#define MPI_INT32_T 4
#define MPI_UINT8_T 1
#define MPI_DOUBLE_COMPLEX 16
#define MPI_C_DOUBLE_COMPLEX 17
#define MPI_CXX_BOOL 18
#define MPI_C_BOOL 18
#define MPI_CHAR 1
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_BOR 4
#define MPI_LOR 5
#define MPI_UNDEFINED (-32766)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_REQUEST_NULL 0

inline int qsref_mpi_type_size(MPI_Datatype t) {
    switch (t) {
    case MPI_BYTE: return 1;
    case MPI_INT: return 4;
    case MPI_FLOAT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_INT64_T: return 8;
    case MPI_UINT64_T: return 8;
    case MPI_UINT: return 4;
    case MPI_DOUBLE_COMPLEX: return 16;
    case MPI_C_DOUBLE_COMPLEX: return 16;
    default: return 1;
    }
}
inline void qsref_mpi_copy(void* dst, const void* src, int count, MPI_Datatype t) {
    if (src == MPI_IN_PLACE || dst == src) return;
    std::memmove(dst, src, (size_t)count * (size_t)qsref_mpi_type_size(t));
}

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Comm_split(MPI_Comm c, int color, int, MPI_Comm* out) { *out = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : c; return 0; }
inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* out) { *out = c; return 0; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) { qsref_mpi_copy(r, s, n, t); return 0; }
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) { qsref_mpi_copy(r, s, n, t); return 0; }
inline int MPI_Iallreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm, MPI_Request* q) { qsref_mpi_copy(r, s, n, t); if (q) *q = 0; return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
inline int MPI_Sendrecv(const void* s, int sn, MPI_Datatype st, int, int, void* r, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { qsref_mpi_copy(r, s, sn, st); return 0; }
inline int MPI_Sendrecv_replace(void*, int, MPI_Datatype, int, int, int, int, MPI_Comm, MPI_Status*) { return 0; }
inline int MPI_Gather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm) { qsref_mpi_copy(r, s, sn, st); return 0; }
inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) { qsref_mpi_copy(r, s, sn, st); return 0; }
inline int MPI_Scatter(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm) { qsref_mpi_copy(r, s, sn, st); return 0; }
inline int MPI_Gatherv(const void* s, int sn, MPI_Datatype st, void* r, const int*, const int* displs, MPI_Datatype, int, MPI_Comm) {
    qsref_mpi_copy((char*)r + (size_t)displs[0] * qsref_mpi_type_size(st), s, sn, st); return 0; }
inline int MPI_Allgatherv(const void* s, int sn, MPI_Datatype st, void* r, const int*, const int* displs, MPI_Datatype, MPI_Comm) {
    if (s == MPI_IN_PLACE) return 0;
    qsref_mpi_copy((char*)r + (size_t)displs[0] * qsref_mpi_type_size(st), s, sn, st); return 0; }
inline int MPI_Scatterv(const void* s, const int*, const int* displs, MPI_Datatype st, void* r, int rn, MPI_Datatype, int, MPI_Comm) {
    qsref_mpi_copy(r, (const char*)s + (size_t)displs[0] * qsref_mpi_type_size(st), rn, st); return 0; }
inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm) {
    qsref_mpi_copy((char*)r + (size_t)rd[0] * qsref_mpi_type_size(st), (const char*)s + (size_t)sd[0] * qsref_mpi_type_size(st), sc[0], st); return 0; }
inline int MPI_Ialltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int* rc, const int* rd, MPI_Datatype rt, MPI_Comm c, MPI_Request* q) {
    if (q) *q = 0;
    return MPI_Alltoallv(s, sc, sd, st, r, rc, rd, rt, c); }
/* point-to-point messages to oneself never occur on the single-rank paths the
   oracle drives; a send or receive is accepted and moves nothing */
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { if (q) *q = 0; return 0; }
inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { if (q) *q = 0; return 0; }
inline double MPI_Wtime() { return 0.0; }
