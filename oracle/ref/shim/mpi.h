/* mpi.h -- single-process stand-in for MPI, used only to compile the
 * reference Grains3D sources as the CPU oracle (test infrastructure).  Rank 0
 * of a world of size 1: collectives copy the send buffer into the receive
 * buffer, point-to-point calls are never reached with one rank, MPI-IO maps
 * onto stdio. */
#ifndef GRAINS_ORACLE_MPI_SHIM_H
#define GRAINS_ORACLE_MPI_SHIM_H
#include <stdio.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Group;
typedef int MPI_Request;
typedef int MPI_Info;
typedef FILE* MPI_File;
typedef long long MPI_Offset;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR, count;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_CHAR 1
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_UNSIGNED_LONG 9
#define MPI_UNSIGNED_SHORT 2
#define MPI_SUM 0
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_LAND 3
#define MPI_INFO_NULL 0
#define MPI_MODE_WRONLY 1
#define MPI_MODE_CREATE 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)

static inline int mpi_shim_size(MPI_Datatype t) {
  return t == MPI_CHAR ? 1 : t == MPI_UNSIGNED_SHORT ? 2 : t == MPI_INT ? 4 : 8;
}
static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Initialized(int* f) { *f = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline double MPI_Wtime() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
static inline int MPI_Abort(MPI_Comm, int) { return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)n * mpi_shim_size(t));
  return 0;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (r && s != r) memmove(r, s, (size_t)n * mpi_shim_size(t));
  return 0;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)n * mpi_shim_size(t));
  return 0;
}
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
  if (r && s != r) memmove(r, s, (size_t)n * mpi_shim_size(t));
  return 0;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
static inline int MPI_Probe(int, int, MPI_Comm, MPI_Status* st) {
  if (st) st->count = 0;
  return 0;
}
static inline int MPI_Get_count(const MPI_Status*, MPI_Datatype, int* c) { *c = 0; return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Type_contiguous(int, MPI_Datatype o, MPI_Datatype* t) { *t = o; return 0; }
static inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
static inline int MPI_Type_free(MPI_Datatype*) { return 0; }
static inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 1; return 0; }
static inline int MPI_Group_incl(MPI_Group, int, const int*, MPI_Group* g) { *g = 1; return 0; }
static inline int MPI_Group_free(MPI_Group*) { return 0; }
static inline int MPI_Comm_create(MPI_Comm c, MPI_Group, MPI_Comm* o) { *o = c; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* o) { *o = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm*) { return 0; }
static inline int MPI_Cart_create(MPI_Comm c, int, const int*, const int*, int, MPI_Comm* o) { *o = c; return 0; }
static inline int MPI_Cart_rank(MPI_Comm, const int*, int* r) { *r = 0; return 0; }
static inline int MPI_Cart_coords(MPI_Comm, int, int n, int* c) {
  for (int i = 0; i < n; ++i) c[i] = 0;
  return 0;
}
static inline int MPI_File_open(MPI_Comm, const char* name, int, MPI_Info, MPI_File* f) {
  *f = fopen(name, "wb");
  return *f ? 0 : 1;
}
static inline int MPI_File_close(MPI_File* f) {
  if (*f) fclose(*f);
  *f = 0;
  return 0;
}
static inline int MPI_File_write(MPI_File f, const void* b, int n, MPI_Datatype t, MPI_Status*) {
  fwrite(b, (size_t)mpi_shim_size(t), (size_t)n, f);
  return 0;
}
static inline int MPI_File_write_at(MPI_File f, MPI_Offset o, const void* b, int n, MPI_Datatype t, MPI_Status*) {
  fseek(f, (long)o, SEEK_SET);
  fwrite(b, (size_t)mpi_shim_size(t), (size_t)n, f);
  return 0;
}
static inline int MPI_File_write_at_all(MPI_File f, MPI_Offset o, const void* b, int n, MPI_Datatype t,
                                        MPI_Status* s) {
  return MPI_File_write_at(f, o, b, n, t, s);
}
#endif
