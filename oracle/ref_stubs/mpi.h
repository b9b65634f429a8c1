/*
 * Single-process MPI subset, written for this project as TEST INFRASTRUCTURE.
 *
 * It exists only so that the reference's header-only CPU path (its MPI
 * backend, bcl/backends/mpi/*.hpp) compiles and runs as one rank in a
 * container without an MPI installation.  The reference then serves as the
 * oracle and the timed CPU baseline for the sparse tile multiply.
 *
 * Semantics: one rank (rank 0, size 1).  An RMA window is a private anonymous
 * mapping (lazily committed, so a multi-GB segment costs nothing until
 * touched).  Rget/Rput are memcpy into/out of that mapping at the given byte
 * displacement; collectives with one participant are copies or no-ops.
 */
#ifndef BCLX_MPI_STUB_H
#define BCLX_MPI_STUB_H

#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>

typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Info;
typedef int MPI_Request;
typedef int MPI_Win;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_THREAD_MULTIPLE 3

/* datatypes: the value encodes the element size in bytes in the low byte */
#define MPI_CHAR               (0x100 | 1)
#define MPI_C_BOOL             (0x200 | 1)
#define MPI_INT8_T             (0x300 | 1)
#define MPI_UINT8_T            (0x400 | 1)
#define MPI_INT16_T            (0x500 | 2)
#define MPI_UINT16_T           (0x600 | 2)
#define MPI_UNSIGNED_SHORT     (0x700 | 2)
#define MPI_INT                (0x800 | 4)
#define MPI_INT32_T            (0x900 | 4)
#define MPI_UINT32_T           (0xa00 | 4)
#define MPI_FLOAT              (0xb00 | 4)
#define MPI_INT64_T            (0xc00 | 8)
#define MPI_UINT64_T           (0xd00 | 8)
#define MPI_UNSIGNED_LONG_LONG (0xe00 | 8)
#define MPI_DOUBLE             (0xf00 | 8)
#define MPI_LONG_DOUBLE        (0x1000 | 16)

#define MPI_SUM  1
#define MPI_BOR  2
#define MPI_BXOR 3
#define MPI_BAND 4
#define MPI_LAND 5
#define MPI_REPLACE 6
#define MPI_NO_OP 7

static inline size_t bclx_stub_type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

/* window bookkeeping: a handful of windows is plenty for one process */
#define BCLX_STUB_MAX_WINS 16
static char* bclx_stub_win_base[BCLX_STUB_MAX_WINS];
static size_t bclx_stub_win_size[BCLX_STUB_MAX_WINS];
static int bclx_stub_initialized = 0;
static int bclx_stub_finalized = 0;

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; bclx_stub_initialized = 1; return 0; }
static inline int MPI_Init_thread(int* argc, char*** argv, int req, int* prov) {
  (void)argc; (void)argv; *prov = req; bclx_stub_initialized = 1; return 0;
}
static inline int MPI_Initialized(int* flag) { *flag = bclx_stub_initialized; return 0; }
static inline int MPI_Finalized(int* flag) { *flag = bclx_stub_finalized; return 0; }
static inline int MPI_Finalize(void) { bclx_stub_finalized = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Info_create(MPI_Info* i) { *i = 1; return 0; }
static inline int MPI_Info_set(MPI_Info i, const char* k, const char* v) { (void)i; (void)k; (void)v; return 0; }
static inline int MPI_Info_free(MPI_Info* i) { *i = MPI_INFO_NULL; return 0; }

static inline int MPI_Win_allocate(MPI_Aint size, int disp_unit, MPI_Info info, MPI_Comm comm,
                                   void* baseptr, MPI_Win* win) {
  (void)disp_unit; (void)info; (void)comm;
  int w = 0;
  while (w < BCLX_STUB_MAX_WINS && bclx_stub_win_base[w] != NULL) w++;
  if (w == BCLX_STUB_MAX_WINS) return 1;
  size_t bytes = size > 0 ? (size_t)size : 1;
  void* p = mmap(NULL, bytes, PROT_READ | PROT_WRITE,
                 MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
  if (p == MAP_FAILED) return 1;
  bclx_stub_win_base[w] = (char*)p;
  bclx_stub_win_size[w] = bytes;
  *(void**)baseptr = p;
  *win = w;
  return 0;
}
static inline int MPI_Win_free(MPI_Win* win) {
  if (bclx_stub_win_base[*win]) munmap(bclx_stub_win_base[*win], bclx_stub_win_size[*win]);
  bclx_stub_win_base[*win] = NULL;
  return 0;
}
static inline int MPI_Win_lock_all(int a, MPI_Win w) { (void)a; (void)w; return 0; }
static inline int MPI_Win_unlock_all(MPI_Win w) { (void)w; return 0; }
static inline int MPI_Win_flush_all(MPI_Win w) { (void)w; return 0; }
static inline int MPI_Win_flush_local(int r, MPI_Win w) { (void)r; (void)w; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

static inline int MPI_Rget(void* dst, int count, MPI_Datatype dt, int rank, MPI_Aint disp,
                           int tcount, MPI_Datatype tdt, MPI_Win win, MPI_Request* req) {
  (void)rank; (void)tcount; (void)tdt;
  memcpy(dst, bclx_stub_win_base[win] + disp, (size_t)count * bclx_stub_type_size(dt));
  *req = 1;
  return 0;
}
static inline int MPI_Rput(const void* src, int count, MPI_Datatype dt, int rank, MPI_Aint disp,
                           int tcount, MPI_Datatype tdt, MPI_Win win, MPI_Request* req) {
  (void)rank; (void)tcount; (void)tdt;
  memcpy(bclx_stub_win_base[win] + disp, src, (size_t)count * bclx_stub_type_size(dt));
  *req = 1;
  return 0;
}
static inline int MPI_Wait(MPI_Request* r, MPI_Status* s) { (void)s; *r = MPI_REQUEST_NULL; return 0; }
static inline int MPI_Test(MPI_Request* r, int* flag, MPI_Status* s) { (void)s; *r = MPI_REQUEST_NULL; *flag = 1; return 0; }
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) { (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Ibcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c, MPI_Request* r) {
  (void)b; (void)n; (void)t; (void)root; (void)c; *r = 1; return 0;
}

/* element-wise op on one element of size/type dt: dst = dst (op) src */
static inline void bclx_stub_apply(void* dst, const void* src, MPI_Datatype dt, MPI_Op op) {
  if (op == MPI_REPLACE) { memcpy(dst, src, bclx_stub_type_size(dt)); return; }
  if (op == MPI_NO_OP) return;
#define BCLX_STUB_OP(T) { T a; T b; memcpy(&a, dst, sizeof(T)); memcpy(&b, src, sizeof(T)); \
    if (op == MPI_SUM) a = (T)(a + b); \
    memcpy(dst, &a, sizeof(T)); return; }
#define BCLX_STUB_IOP(T) { T a; T b; memcpy(&a, dst, sizeof(T)); memcpy(&b, src, sizeof(T)); \
    if (op == MPI_SUM) a = (T)(a + b); else if (op == MPI_BOR) a = (T)(a | b); \
    else if (op == MPI_BXOR) a = (T)(a ^ b); else if (op == MPI_BAND) a = (T)(a & b); \
    else if (op == MPI_LAND) a = (T)(a && b); \
    memcpy(dst, &a, sizeof(T)); return; }
  switch (dt) {
    case MPI_FLOAT: BCLX_STUB_OP(float)
    case MPI_DOUBLE: BCLX_STUB_OP(double)
    case MPI_INT: case MPI_INT32_T: BCLX_STUB_IOP(int32_t)
    case MPI_UINT32_T: BCLX_STUB_IOP(uint32_t)
    case MPI_INT64_T: BCLX_STUB_IOP(int64_t)
    case MPI_UINT64_T: case MPI_UNSIGNED_LONG_LONG: BCLX_STUB_IOP(uint64_t)
    case MPI_INT16_T: BCLX_STUB_IOP(int16_t)
    case MPI_UINT16_T: case MPI_UNSIGNED_SHORT: BCLX_STUB_IOP(uint16_t)
    case MPI_INT8_T: BCLX_STUB_IOP(int8_t)
    default: BCLX_STUB_IOP(uint8_t)
  }
#undef BCLX_STUB_OP
#undef BCLX_STUB_IOP
}

static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  (void)op; (void)c;
  memcpy(r, s, (size_t)n * bclx_stub_type_size(t));
  return 0;
}
static inline int MPI_Rget_accumulate(const void* origin, int ocount, MPI_Datatype odt,
                                      void* result, int rcount, MPI_Datatype rdt,
                                      int rank, MPI_Aint disp, int tcount, MPI_Datatype tdt,
                                      MPI_Op op, MPI_Win win, MPI_Request* req) {
  (void)rcount; (void)rdt; (void)rank; (void)tcount; (void)tdt;
  size_t es = bclx_stub_type_size(odt);
  char* target = bclx_stub_win_base[win] + disp;
  memcpy(result, target, (size_t)ocount * es);
  for (int i = 0; i < ocount; i++) bclx_stub_apply(target + i * es, (const char*)origin + i * es, odt, op);
  *req = 1;
  return 0;
}
static inline int MPI_Compare_and_swap(const void* newv, const void* cmpv, void* result,
                                       MPI_Datatype dt, int rank, MPI_Aint disp, MPI_Win win) {
  (void)rank;
  size_t es = bclx_stub_type_size(dt);
  char* target = bclx_stub_win_base[win] + disp;
  memcpy(result, target, es);
  if (memcmp(target, cmpv, es) == 0) memcpy(target, newv, es);
  return 0;
}
static inline int MPI_Comm_group(MPI_Comm c, MPI_Group* g) { (void)c; *g = 1; return 0; }
static inline int MPI_Group_incl(MPI_Group g, int n, const int* r, MPI_Group* ng) { (void)g; (void)n; (void)r; *ng = 1; return 0; }
static inline int MPI_Group_free(MPI_Group* g) { *g = 0; return 0; }
static inline int MPI_Comm_create(MPI_Comm c, MPI_Group g, MPI_Comm* nc) { (void)c; (void)g; *nc = 2; return 0; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Alloc_mem(MPI_Aint size, MPI_Info info, void* baseptr) {
  (void)info; *(void**)baseptr = malloc((size_t)size); return 0;
}
static inline int MPI_Free_mem(void* p) { free(p); return 0; }

#endif
