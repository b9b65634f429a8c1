/*
 * Multi-process MPI subset over shared memory, written for this project as
 * TEST INFRASTRUCTURE.
 *
 * It lets the reference's header-only MPI backend (the bcl/backends/mpi
 * headers) run as several ranks on one host without an MPI installation, so that the
 * reference's own distributed BCL::gemm (bcl/containers/algorithms/
 * spgemm.hpp:153-242: block-cyclic tiles, remote tile fetches, barriers,
 * pointer broadcasts) runs as written.  The ranks are separate processes
 * started by a launcher (oracle.py: run_ref_mp) with
 *   BCLX_STUB_RANK, BCLX_STUB_SIZE  this rank and the number of ranks,
 *   BCLX_STUB_DIR                   a fresh directory shared by the ranks
 *                                   (tmpfs: /dev/shm),
 *   BCLX_STUB_TIMEOUT               seconds a rank waits in a collective
 *                                   before it aborts (default 300).
 *
 * Semantics:
 *   - an RMA window is one file per rank in BCLX_STUB_DIR, mapped shared by
 *     every rank (sparse: a multi-GB segment costs only the pages touched);
 *     Rget / Rput are memcpy from / to the target rank's mapping at the byte
 *     displacement and complete at once (Wait and Test return immediately);
 *   - Barrier is a generation barrier on a shared control block; every
 *     collective and every flush is a full memory fence;
 *   - Bcast / Ibcast stage the data through the control block (1 MiB at a
 *     time, two barriers per piece); Allreduce folds the ranks' values in
 *     rank order (at most 64 bytes per rank);
 *   - Rget_accumulate and Compare_and_swap run under one shared lock;
 *   - sub-communicators (Comm_create) are kept as rank lists; collectives on
 *     one that is not the whole world in order abort.
 * Only the calls the reference's MPI backend makes are provided.
 */
#ifndef BCLX_MPI_STUB_MP_H
#define BCLX_MPI_STUB_MP_H

#include <fcntl.h>
#include <sched.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <time.h>
#include <unistd.h>

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

#define BCLX_MP_MAX_RANKS 256
#define BCLX_MP_MAX_WINS 16
#define BCLX_MP_MAX_GROUPS 64
#define BCLX_MP_SLOT_BYTES 64
#define BCLX_MP_BCAST_BYTES (1u << 20)

typedef struct {
  uint64_t count; /* barrier arrivals in the current generation */
  uint64_t gen;   /* barrier generation */
  uint64_t lock;  /* accumulate / compare-and-swap */
  uint64_t pad[13];
  unsigned char slots[BCLX_MP_MAX_RANKS][BCLX_MP_SLOT_BYTES];
  unsigned char bcast[BCLX_MP_BCAST_BYTES];
} bclx_mp_ctl_t;

static int bclx_mp_rank = 0, bclx_mp_size = 1;
static char bclx_mp_dir[4096];
static double bclx_mp_timeout = 300.0;
static bclx_mp_ctl_t* bclx_mp_ctl = NULL;
static int bclx_mp_initialized = 0, bclx_mp_finalized = 0;
static int bclx_mp_nwins = 0;
static char* bclx_mp_win_base[BCLX_MP_MAX_WINS][BCLX_MP_MAX_RANKS];
static size_t bclx_mp_win_bytes[BCLX_MP_MAX_WINS];
/* groups and communicators: rank lists (id 1 is the world) */
static int bclx_mp_ngroups = 2;
static int bclx_mp_group_n[BCLX_MP_MAX_GROUPS];
static int* bclx_mp_group_ranks[BCLX_MP_MAX_GROUPS];

static inline void bclx_mp_die(const char* what) {
  fprintf(stderr, "mpi stub (rank %d of %d): %s\n", bclx_mp_rank, bclx_mp_size, what);
  fflush(stderr);
  abort();
}

static inline double bclx_mp_now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static inline void bclx_mp_fence(void) { __atomic_thread_fence(__ATOMIC_SEQ_CST); }

static inline void bclx_mp_barrier(void) {
  bclx_mp_fence();
  if (bclx_mp_size == 1) return;
  const uint64_t gen = __atomic_load_n(&bclx_mp_ctl->gen, __ATOMIC_ACQUIRE);
  if (__atomic_add_fetch(&bclx_mp_ctl->count, 1, __ATOMIC_ACQ_REL) == (uint64_t)bclx_mp_size) {
    __atomic_store_n(&bclx_mp_ctl->count, 0, __ATOMIC_RELAXED);
    __atomic_store_n(&bclx_mp_ctl->gen, gen + 1, __ATOMIC_RELEASE);
  } else {
    const double t0 = bclx_mp_now();
    unsigned spins = 0;
    while (__atomic_load_n(&bclx_mp_ctl->gen, __ATOMIC_ACQUIRE) == gen) {
      if (++spins > 64) sched_yield();
      if ((spins & 1023) == 0 && bclx_mp_now() - t0 > bclx_mp_timeout) bclx_mp_die("barrier timed out");
    }
  }
  bclx_mp_fence();
}

static inline void bclx_mp_lock(void) {
  const double t0 = bclx_mp_now();
  unsigned spins = 0;
  while (__atomic_exchange_n(&bclx_mp_ctl->lock, 1, __ATOMIC_ACQUIRE) != 0) {
    if (++spins > 64) sched_yield();
    if ((spins & 1023) == 0 && bclx_mp_now() - t0 > bclx_mp_timeout) bclx_mp_die("lock timed out");
  }
}
static inline void bclx_mp_unlock(void) { __atomic_store_n(&bclx_mp_ctl->lock, 0, __ATOMIC_RELEASE); }

static inline void* bclx_mp_map(const char* path, size_t bytes, int create) {
  const int fd = open(path, O_RDWR | (create ? O_CREAT : 0), 0600);
  if (fd < 0) bclx_mp_die("cannot open a shared file");
  if (create && ftruncate(fd, (off_t)bytes) != 0) bclx_mp_die("cannot size a shared file");
  void* p = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_NORESERVE, fd, 0);
  close(fd);
  if (p == MAP_FAILED) bclx_mp_die("cannot map a shared file");
  return p;
}

static inline int bclx_mp_env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return v && *v ? atoi(v) : dflt;
}

static inline int MPI_Init(int* argc, char*** argv) {
  (void)argc; (void)argv;
  bclx_mp_rank = bclx_mp_env_int("BCLX_STUB_RANK", 0);
  bclx_mp_size = bclx_mp_env_int("BCLX_STUB_SIZE", 1);
  const char* t = getenv("BCLX_STUB_TIMEOUT");
  if (t && *t) bclx_mp_timeout = atof(t);
  if (bclx_mp_size < 1 || bclx_mp_size > BCLX_MP_MAX_RANKS || bclx_mp_rank < 0 || bclx_mp_rank >= bclx_mp_size)
    bclx_mp_die("bad BCLX_STUB_RANK / BCLX_STUB_SIZE");
  const char* d = getenv("BCLX_STUB_DIR");
  if (!d || !*d) {
    if (bclx_mp_size > 1) bclx_mp_die("BCLX_STUB_DIR is not set");
    d = "/tmp";
  }
  snprintf(bclx_mp_dir, sizeof(bclx_mp_dir), "%s", d);
  char path[4200];
  snprintf(path, sizeof(path), "%s/ctl", bclx_mp_dir);
  if (bclx_mp_size > 1) {
    /* every rank sizes the same file to the same length: the first one
       creates it zero-filled, the others change nothing */
    bclx_mp_ctl = (bclx_mp_ctl_t*)bclx_mp_map(path, sizeof(bclx_mp_ctl_t), 1);
  } else {
    bclx_mp_ctl = (bclx_mp_ctl_t*)calloc(1, sizeof(bclx_mp_ctl_t));
  }
  bclx_mp_group_n[1] = bclx_mp_size;
  bclx_mp_group_ranks[1] = (int*)malloc(sizeof(int) * (size_t)bclx_mp_size);
  for (int r = 0; r < bclx_mp_size; r++) bclx_mp_group_ranks[1][r] = r;
  bclx_mp_initialized = 1;
  bclx_mp_barrier();
  return 0;
}
static inline int MPI_Init_thread(int* argc, char*** argv, int req, int* prov) {
  *prov = req;
  return MPI_Init(argc, argv);
}
static inline int MPI_Initialized(int* flag) { *flag = bclx_mp_initialized; return 0; }
static inline int MPI_Finalized(int* flag) { *flag = bclx_mp_finalized; return 0; }
static inline int MPI_Finalize(void) {
  bclx_mp_barrier();
  bclx_mp_finalized = 1;
  return 0;
}

/* the group of a communicator (world, or one made by MPI_Comm_create) */
static inline int bclx_mp_comm_group(MPI_Comm c) {
  if (c <= 0 || c >= bclx_mp_ngroups || !bclx_mp_group_ranks[c]) bclx_mp_die("unknown communicator");
  return c;
}
/* collectives run on the world; a communicator equal to it is accepted */
static inline void bclx_mp_world_only(MPI_Comm c) {
  const int g = bclx_mp_comm_group(c);
  if (bclx_mp_group_n[g] != bclx_mp_size) bclx_mp_die("collective on a sub-communicator");
  for (int r = 0; r < bclx_mp_size; r++)
    if (bclx_mp_group_ranks[g][r] != r) bclx_mp_die("collective on a reordered communicator");
}
static inline int MPI_Comm_rank(MPI_Comm c, int* r) {
  const int g = bclx_mp_comm_group(c);
  for (int i = 0; i < bclx_mp_group_n[g]; i++)
    if (bclx_mp_group_ranks[g][i] == bclx_mp_rank) { *r = i; return 0; }
  bclx_mp_die("rank not in communicator");
  return 1;
}
static inline int MPI_Comm_size(MPI_Comm c, int* s) { *s = bclx_mp_group_n[bclx_mp_comm_group(c)]; return 0; }
static inline int MPI_Info_create(MPI_Info* i) { *i = 1; return 0; }
static inline int MPI_Info_set(MPI_Info i, const char* k, const char* v) { (void)i; (void)k; (void)v; return 0; }
static inline int MPI_Info_free(MPI_Info* i) { *i = MPI_INFO_NULL; return 0; }

static inline int MPI_Barrier(MPI_Comm c) {
  bclx_mp_world_only(c);
  bclx_mp_barrier();
  return 0;
}

/* collective: every rank maps its own file, then every other rank's */
static inline int MPI_Win_allocate(MPI_Aint size, int disp_unit, MPI_Info info, MPI_Comm comm,
                                   void* baseptr, MPI_Win* win) {
  (void)disp_unit; (void)info;
  bclx_mp_world_only(comm);
  if (bclx_mp_nwins == BCLX_MP_MAX_WINS) bclx_mp_die("too many windows");
  const int w = bclx_mp_nwins++;
  const size_t bytes = size > 0 ? (size_t)size : 1;
  char path[4200];
  if (bclx_mp_size == 1) {
    void* p = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (p == MAP_FAILED) bclx_mp_die("cannot map a window");
    bclx_mp_win_base[w][0] = (char*)p;
  } else {
    snprintf(path, sizeof(path), "%s/w%d_r%d", bclx_mp_dir, w, bclx_mp_rank);
    bclx_mp_win_base[w][bclx_mp_rank] = (char*)bclx_mp_map(path, bytes, 1);
    bclx_mp_barrier();
    for (int r = 0; r < bclx_mp_size; r++) {
      if (r == bclx_mp_rank) continue;
      snprintf(path, sizeof(path), "%s/w%d_r%d", bclx_mp_dir, w, r);
      bclx_mp_win_base[w][r] = (char*)bclx_mp_map(path, bytes, 0);
    }
    bclx_mp_barrier();
  }
  bclx_mp_win_bytes[w] = bytes;
  *(void**)baseptr = bclx_mp_win_base[w][bclx_mp_rank];
  *win = w;
  return 0;
}
static inline int MPI_Win_free(MPI_Win* win) {
  bclx_mp_barrier();
  for (int r = 0; r < bclx_mp_size; r++)
    if (bclx_mp_win_base[*win][r]) munmap(bclx_mp_win_base[*win][r], bclx_mp_win_bytes[*win]);
  if (bclx_mp_size > 1) {
    char path[4200];
    snprintf(path, sizeof(path), "%s/w%d_r%d", bclx_mp_dir, *win, bclx_mp_rank);
    unlink(path);
  }
  memset(bclx_mp_win_base[*win], 0, sizeof(bclx_mp_win_base[*win]));
  return 0;
}
static inline int MPI_Win_lock_all(int a, MPI_Win w) { (void)a; (void)w; bclx_mp_fence(); return 0; }
static inline int MPI_Win_unlock_all(MPI_Win w) { (void)w; bclx_mp_fence(); return 0; }
static inline int MPI_Win_flush_all(MPI_Win w) { (void)w; bclx_mp_fence(); return 0; }
static inline int MPI_Win_flush_local(int r, MPI_Win w) { (void)r; (void)w; bclx_mp_fence(); return 0; }

static inline char* bclx_mp_target(MPI_Win win, int rank, MPI_Aint disp, size_t bytes) {
  if (win < 0 || win >= bclx_mp_nwins || rank < 0 || rank >= bclx_mp_size || !bclx_mp_win_base[win][rank])
    bclx_mp_die("bad window or rank");
  if (disp < 0 || (size_t)disp + bytes > bclx_mp_win_bytes[win]) bclx_mp_die("access outside the window");
  return bclx_mp_win_base[win][rank] + disp;
}

static inline int MPI_Rget(void* dst, int count, MPI_Datatype dt, int rank, MPI_Aint disp,
                           int tcount, MPI_Datatype tdt, MPI_Win win, MPI_Request* req) {
  (void)tcount; (void)tdt;
  const size_t bytes = (size_t)count * bclx_stub_type_size(dt);
  memcpy(dst, bclx_mp_target(win, rank, disp, bytes), bytes);
  *req = 1;
  return 0;
}
static inline int MPI_Rput(const void* src, int count, MPI_Datatype dt, int rank, MPI_Aint disp,
                           int tcount, MPI_Datatype tdt, MPI_Win win, MPI_Request* req) {
  (void)tcount; (void)tdt;
  const size_t bytes = (size_t)count * bclx_stub_type_size(dt);
  memcpy(bclx_mp_target(win, rank, disp, bytes), src, bytes);
  *req = 1;
  return 0;
}
static inline int MPI_Wait(MPI_Request* r, MPI_Status* s) { (void)s; *r = MPI_REQUEST_NULL; return 0; }
static inline int MPI_Test(MPI_Request* r, int* flag, MPI_Status* s) { (void)s; *r = MPI_REQUEST_NULL; *flag = 1; return 0; }

static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  bclx_mp_world_only(c);
  if (bclx_mp_size == 1) return 0;
  const size_t bytes = (size_t)n * bclx_stub_type_size(t);
  size_t off = 0;
  do {
    const size_t len = bytes - off < BCLX_MP_BCAST_BYTES ? bytes - off : BCLX_MP_BCAST_BYTES;
    bclx_mp_barrier(); /* the staging area's previous contents have been read */
    if (bclx_mp_rank == root) memcpy(bclx_mp_ctl->bcast, (char*)b + off, len);
    bclx_mp_barrier();
    if (bclx_mp_rank != root) memcpy((char*)b + off, bclx_mp_ctl->bcast, len);
    off += len;
  } while (off < bytes);
  return 0;
}
static inline int MPI_Ibcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c, MPI_Request* r) {
  *r = 1;
  return MPI_Bcast(b, n, t, root, c);
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
  bclx_mp_world_only(c);
  const size_t es = bclx_stub_type_size(t), bytes = (size_t)n * es;
  if (bclx_mp_size == 1) { memcpy(r, s, bytes); return 0; }
  if (bytes > BCLX_MP_SLOT_BYTES) bclx_mp_die("allreduce larger than a slot");
  memcpy(bclx_mp_ctl->slots[bclx_mp_rank], s, bytes);
  bclx_mp_barrier();
  unsigned char acc[BCLX_MP_SLOT_BYTES];
  memcpy(acc, bclx_mp_ctl->slots[0], bytes);
  for (int q = 1; q < bclx_mp_size; q++)
    for (int i = 0; i < n; i++) bclx_stub_apply(acc + i * es, bclx_mp_ctl->slots[q] + i * es, t, op);
  bclx_mp_barrier(); /* every rank has read the slots */
  memcpy(r, acc, bytes);
  return 0;
}
static inline int MPI_Rget_accumulate(const void* origin, int ocount, MPI_Datatype odt,
                                      void* result, int rcount, MPI_Datatype rdt,
                                      int rank, MPI_Aint disp, int tcount, MPI_Datatype tdt,
                                      MPI_Op op, MPI_Win win, MPI_Request* req) {
  (void)rcount; (void)rdt; (void)tcount; (void)tdt;
  const size_t es = bclx_stub_type_size(odt);
  char* target = bclx_mp_target(win, rank, disp, (size_t)ocount * es);
  bclx_mp_lock();
  memcpy(result, target, (size_t)ocount * es);
  for (int i = 0; i < ocount; i++) bclx_stub_apply(target + i * es, (const char*)origin + i * es, odt, op);
  bclx_mp_unlock();
  *req = 1;
  return 0;
}
static inline int MPI_Compare_and_swap(const void* newv, const void* cmpv, void* result,
                                       MPI_Datatype dt, int rank, MPI_Aint disp, MPI_Win win) {
  const size_t es = bclx_stub_type_size(dt);
  char* target = bclx_mp_target(win, rank, disp, es);
  bclx_mp_lock();
  memcpy(result, target, es);
  if (memcmp(target, cmpv, es) == 0) memcpy(target, newv, es);
  bclx_mp_unlock();
  return 0;
}
static inline int MPI_Comm_group(MPI_Comm c, MPI_Group* g) { *g = bclx_mp_comm_group(c); return 0; }
/* a group: the listed ranks of group g, in that order (kept per process) */
static inline int MPI_Group_incl(MPI_Group g, int n, const int* r, MPI_Group* ng) {
  if (bclx_mp_ngroups == BCLX_MP_MAX_GROUPS) bclx_mp_die("too many groups");
  const int id = bclx_mp_ngroups++;
  bclx_mp_group_n[id] = n;
  bclx_mp_group_ranks[id] = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) bclx_mp_group_ranks[id][i] = bclx_mp_group_ranks[g][r[i]];
  *ng = id;
  return 0;
}
static inline int MPI_Group_free(MPI_Group* g) { *g = 0; return 0; }
/* collective over c: members get a communicator with the group's ranks */
static inline int MPI_Comm_create(MPI_Comm c, MPI_Group g, MPI_Comm* nc) {
  bclx_mp_world_only(c);
  bclx_mp_barrier();
  *nc = MPI_COMM_NULL;
  for (int i = 0; i < bclx_mp_group_n[g]; i++)
    if (bclx_mp_group_ranks[g][i] == bclx_mp_rank) *nc = g;
  return 0;
}
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Alloc_mem(MPI_Aint size, MPI_Info info, void* baseptr) {
  (void)info; *(void**)baseptr = malloc((size_t)size); return 0;
}
static inline int MPI_Free_mem(void* p) { free(p); return 0; }

#endif
