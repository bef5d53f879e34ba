/* Single-rank stand-in for the MPI C API, written for this project so that the
 * reference library's CPU path can be compiled here without an MPI install.
 * Every communicator has one rank (rank 0).  Collectives copy the send buffer
 * into the receive buffer; point-to-point calls are never reached on one rank
 * (the halo refresh of a single node is a local periodic copy) and return 0.
 * A datatype handle encodes its byte size as (size << 8) | id.  This file is
 * test infrastructure for the oracle only. */
#pragma once
#include <stddef.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long MPI_Aint;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int count_lo;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_INFO_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_MAX_ERROR_STRING 256
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_REQUEST_NULL 0
#define MPI_IN_PLACE ((void*)1)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

#define QSHIM_DT(size, id) (((size) << 8) | (id))
#define MPI_DATATYPE_NULL 0
#define MPI_BYTE QSHIM_DT(1, 1)
#define MPI_CHAR QSHIM_DT(1, 2)
#define MPI_UNSIGNED_CHAR QSHIM_DT(1, 3)
#define MPI_INT QSHIM_DT(4, 4)
#define MPI_UNSIGNED QSHIM_DT(4, 5)
#define MPI_LONG QSHIM_DT(8, 6)
#define MPI_UNSIGNED_LONG QSHIM_DT(8, 7)
#define MPI_LONG_LONG QSHIM_DT(8, 8)
#define MPI_UNSIGNED_LONG_LONG QSHIM_DT(8, 9)
#define MPI_FLOAT QSHIM_DT(4, 10)
#define MPI_DOUBLE QSHIM_DT(8, 11)
#define MPI_LOGICAL QSHIM_DT(4, 12)
#define MPI_INT64_T QSHIM_DT(8, 13)
#define MPI_UINT64_T QSHIM_DT(8, 14)
#define MPI_INT32_T QSHIM_DT(4, 15)
#define MPI_UINT32_T QSHIM_DT(4, 16)
#define MPI_INT8_T QSHIM_DT(1, 17)
#define MPI_UINT8_T QSHIM_DT(1, 18)
#define MPI_INT16_T QSHIM_DT(2, 21)
#define MPI_UINT16_T QSHIM_DT(2, 22)
#define MPI_SHORT QSHIM_DT(2, 23)
#define MPI_UNSIGNED_SHORT QSHIM_DT(2, 24)
#define MPI_C_DOUBLE_COMPLEX QSHIM_DT(16, 19)
#define MPI_C_FLOAT_COMPLEX QSHIM_DT(8, 20)

#define MPI_OP_NULL 0
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_PROD 4
#define MPI_BXOR 5
#define MPI_BOR 6
#define MPI_BAND 7
#define MPI_LAND 8
#define MPI_LOR 9

static inline int qshim_size(MPI_Datatype t) { return t >> 8; }
static inline void qshim_copy(const void* s, void* r, int count, MPI_Datatype t)
{
  if (s == MPI_IN_PLACE || s == r || count <= 0) return;
  memmove(r, s, (size_t)count * (size_t)qshim_size(t));
}

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Init_thread(int*, char***, int, int* provided)
{
  if (provided) *provided = MPI_THREAD_MULTIPLE;
  return 0;
}
static inline int MPI_Initialized(int* flag) { *flag = 1; return 0; }
static inline int MPI_Finalized(int* flag) { *flag = 0; return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Abort(MPI_Comm, int) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* n) { *n = c; return 0; }
static inline int MPI_Comm_split_type(MPI_Comm c, int, int, MPI_Info, MPI_Comm* n) { *n = c; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* n) { *n = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm*) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Error_string(int, char* s, int* len) { s[0] = 0; *len = 0; return 0; }
static inline int MPI_Get_processor_name(char* s, int* len) { strcpy(s, "oracle"); *len = 6; return 0; }
static inline int MPI_Dims_create(int, int nd, int* dims)
{
  for (int i = 0; i < nd; ++i) if (dims[i] == 0) dims[i] = 1;
  return 0;
}
static inline int MPI_Type_size(MPI_Datatype t, int* s) { *s = qshim_size(t); return 0; }
static inline int MPI_Type_contiguous(int n, MPI_Datatype old, MPI_Datatype* t)
{
  *t = QSHIM_DT(n * qshim_size(old), 63);
  return 0;
}
static inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
static inline int MPI_Type_free(MPI_Datatype* t) { *t = 0; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{ qshim_copy(s, r, n, t); return 0; }
static inline int MPI_Iallreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm, MPI_Request* q)
{ qshim_copy(s, r, n, t); *q = 0; return 0; }
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{ qshim_copy(s, r, n, t); return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm)
{ qshim_copy(s, r, n, t); return 0; }
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm)
{ if (r) qshim_copy(s, r, n, t); return 0; }
static inline int MPI_Scatter(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm)
{ qshim_copy(s, r, n, t); return 0; }
static inline int MPI_Alltoall(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm)
{ qshim_copy(s, r, n, t); return 0; }
static inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r,
                                const int*, const int* rd, MPI_Datatype, MPI_Comm)
{
  const int sz = qshim_size(st);
  if (s != MPI_IN_PLACE) memmove((char*)r + (size_t)rd[0] * sz, (const char*)s + (size_t)sd[0] * sz, (size_t)sc[0] * sz);
  return 0;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Sendrecv(const void* s, int n, MPI_Datatype t, int, int, void* r, int, MPI_Datatype, int, int,
                               MPI_Comm, MPI_Status*)
{ qshim_copy(s, r, n, t); return 0; }
static inline double MPI_Wtime() { return 0.0; }
