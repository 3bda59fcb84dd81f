/*
 * Single-process stand-in for the handful of MPI calls the reference's
 * hot-path sources make.  Test infrastructure only: it exists so that the
 * reference's own C++ can be compiled unmodified (apart from the recorded
 * patch list) and executed on one host as the oracle.
 *
 * The reference decomposes x into slabs, one per rank (Mpi_division.h:7-31),
 * and treats rank 0 / rank nproc-1 specially (inflow/outflow stencils,
 * characteristic boundaries, ghost zeroing).  Running it as "rank 1 of 3"
 * makes every routine take its interior-rank path, and turning every
 * MPI_Sendrecv whose two peers are real ranks into a self-copy makes the
 * 3-plane Q halo (main.cpp:167-200) and the lagged 1-plane NL/NR halo
 * (Dual_time_stepping.cpp:942-976) exactly periodic in x.  Reductions are
 * identities (one participant), broadcasts are no-ops.
 *
 * MPI-IO is backed by pread() so Initial_condition.cpp:111-236 can read a
 * restart file written in its own layout.
 */
#ifndef CGLI_ORACLE_MPI_STUB_H
#define CGLI_ORACLE_MPI_STUB_H

#include <string.h>
#include <stdio.h>
#include <fcntl.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef struct { int fd; } *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_SUM 1
#define MPI_PROC_NULL (-2)
#define MPI_MODE_RDONLY 1
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

/* rank/size the reference sees; set by the harness before any call */
extern int cgli_stub_rank;
extern int cgli_stub_size;
/* path substituted for the reference's hard-wired "initial.bin" */
extern char cgli_stub_initial_path[4096];

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = cgli_stub_size; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = cgli_stub_rank; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }

static inline int cgli_stub_bytes(MPI_Datatype t) { return t; }

/* Both peers real -> the periodic self-copy; either peer MPI_PROC_NULL ->
 * nothing is received (MPI semantics for a null source). */
static inline int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype st, int dest, int,
                               void *rbuf, int rcount, MPI_Datatype rt, int source, int,
                               MPI_Comm, MPI_Status *) {
  (void)rcount; (void)rt;
  if (dest != MPI_PROC_NULL && source != MPI_PROC_NULL && sbuf != rbuf)
    memmove(rbuf, sbuf, (size_t)scount * (size_t)cgli_stub_bytes(st));
  return 0;
}

static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)n * (size_t)cgli_stub_bytes(t));
  return 0;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)n * (size_t)cgli_stub_bytes(t));
  return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }

static inline int MPI_File_open(MPI_Comm, const char *name, int, MPI_Info, MPI_File *fh) {
  static struct { int fd; } slot;
  const char *path = (strcmp(name, "initial.bin") == 0 && cgli_stub_initial_path[0])
                         ? cgli_stub_initial_path : name;
  slot.fd = open(path, O_RDONLY);
  if (slot.fd < 0) { fprintf(stderr, "mpi stub: cannot open %s\n", path); }
  *fh = (MPI_File)&slot;
  return slot.fd < 0;
}
static inline int MPI_File_read_at_all(MPI_File fh, MPI_Offset off, void *buf, int n,
                                       MPI_Datatype t, MPI_Status *) {
  size_t want = (size_t)n * (size_t)cgli_stub_bytes(t);
  ssize_t got = pread(fh->fd, buf, want, (off_t)off);
  return got == (ssize_t)want ? 0 : 1;
}
static inline int MPI_File_close(MPI_File *fh) { close((*fh)->fd); return 0; }

#endif
