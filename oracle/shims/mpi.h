/*
 * mpi.h -- single-rank stand-in for MPI, used only to compile the reference program
 * (fvm_mpi/src) as the test oracle in oracle/_ref.  TEST INFRASTRUCTURE ONLY.
 *
 * One rank: every neighbour is MPI_PROC_NULL, collectives copy their input to their
 * output, point-to-point calls with MPI_PROC_NULL do nothing.
 */
#ifndef CSP_MPI_STUB_H
#define CSP_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_PROC_NULL (-1)
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0

/* datatypes: the value is the element size in bytes (vector types: registered below) */
#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 1
#define MPI_BYTE 1
#define MPI_SHORT 2
#define MPI_UNSIGNED_SHORT 2
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 4
#define MPI_LONG 8
#define MPI_UNSIGNED_LONG 8
#define MPI_LONG_LONG 8
#define MPI_DOUBLE 8

#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3

static inline int csp_mpi_size(MPI_Datatype t) { return t > 0 && t <= 8 ? t : 8; }

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; fflush(stdout); exit(code); return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Cart_create(MPI_Comm c, int nd, const int* dims, const int* periods, int reorder, MPI_Comm* out) {
  (void)nd; (void)dims; (void)periods; (void)reorder; *out = c; return 0;
}
static inline int MPI_Cart_get(MPI_Comm c, int nd, int* dims, int* periods, int* coords) {
  (void)c;
  for (int i = 0; i < nd; i++) { if (dims[i] < 1) dims[i] = 1; periods[i] = 0; coords[i] = 0; }
  return 0;
}
static inline int MPI_Cart_shift(MPI_Comm c, int dir, int disp, int* src, int* dst) {
  (void)c; (void)dir; (void)disp; *src = MPI_PROC_NULL; *dst = MPI_PROC_NULL; return 0;
}
static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request* r) {
  (void)b; (void)n; (void)t; (void)dst; (void)tag; (void)c; *r = 0; return 0;
}
static inline int MPI_Irecv(void* b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request* r) {
  (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c; *r = 0; return 0;
}
static inline int MPI_Waitall(int n, MPI_Request* r, MPI_Status* s) { (void)n; (void)r; (void)s; return 0; }
static inline int MPI_Gather(const void* sb, int sc, MPI_Datatype st, void* rb, int rc, MPI_Datatype rt, int root,
                             MPI_Comm c) {
  (void)rc; (void)rt; (void)root; (void)c;
  if (rb && sb && sc > 0) memmove(rb, sb, (size_t)sc * csp_mpi_size(st));
  return 0;
}
static inline int MPI_Gatherv(const void* sb, int sc, MPI_Datatype st, void* rb, const int* rcs, const int* displs,
                              MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rcs; (void)root; (void)c;
  if (rb && sb && sc > 0) memmove((char*)rb + (size_t)displs[0] * csp_mpi_size(rt), sb, (size_t)sc * csp_mpi_size(st));
  return 0;
}
static inline int MPI_Scatter(const void* sb, int sc, MPI_Datatype st, void* rb, int rc, MPI_Datatype rt, int root,
                              MPI_Comm c) {
  (void)sc; (void)st; (void)root; (void)c;
  if (rb && sb && rc > 0) memmove(rb, sb, (size_t)rc * csp_mpi_size(rt));
  return 0;
}
static inline int MPI_Scatterv(const void* sb, const int* scs, const int* displs, MPI_Datatype st, void* rb, int rc,
                               MPI_Datatype rt, int root, MPI_Comm c) {
  (void)scs; (void)root; (void)c;
  if (rb && sb && rc > 0) memmove(rb, (const char*)sb + (size_t)displs[0] * csp_mpi_size(st), (size_t)rc * csp_mpi_size(rt));
  return 0;
}
static inline int MPI_Reduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c) {
  (void)op; (void)root; (void)c;
  if (rb && sb && n > 0) memmove(rb, sb, (size_t)n * csp_mpi_size(t));
  return 0;
}
static inline int MPI_Allreduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  (void)op; (void)c;
  if (rb && sb && n > 0) memmove(rb, sb, (size_t)n * csp_mpi_size(t));
  return 0;
}
static inline int MPI_Type_vector(int count, int len, int stride, MPI_Datatype old, MPI_Datatype* out) {
  (void)count; (void)len; (void)stride; *out = old; return 0;
}
static inline int MPI_Type_commit(MPI_Datatype* t) { (void)t; return 0; }
static inline int MPI_Type_free(MPI_Datatype* t) { (void)t; return 0; }

#endif
