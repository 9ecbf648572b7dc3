/*
 * One-rank stand-in for <mpi.h>, used only to compile the GAMMA reference
 * sources into the CPU oracle (oracle/_ref).  TEST INFRASTRUCTURE, not product.
 *
 * The 1D reference path never talks to another rank (src/environment.cpp:17
 * refuses worldsize != 1 in 1D), so every call below behaves as it would under
 * `mpirun -n 1`: size 1, rank 0, collectives copy their input, and the
 * point-to-point calls (reachable only with >1 rank, src/Dimensions/2d.cpp:108-238)
 * abort loudly.
 *
 * Call sites covered: src/mpisetup.cpp:18-95, src/simu.cpp, src/main.cpp:150,
 * src/Dimensions/2d.cpp:129-204,966-967, src/IO/text2d.cpp:156-281.
 */
#ifndef GAMMA_ORACLE_SHIM_MPI_H
#define GAMMA_ORACLE_SHIM_MPI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef ptrdiff_t MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0

#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_LONG 3
#define MPI_CHAR 4

#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3

static inline size_t gamma_shim_mpi_size(MPI_Datatype t) {
  switch (t) {
    case MPI_INT: return sizeof(int);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_LONG: return sizeof(long);
    case MPI_CHAR: return 1;
    default: return 0;
  }
}

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Comm_split_type(MPI_Comm c, int type, int key, MPI_Info info, MPI_Comm *out) {
  (void)type; (void)key; (void)info; *out = c; return 0;
}
/* With one rank every reduction is the identity. */
static inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  (void)op; (void)c;
  if (in != out) memcpy(out, in, (size_t)n * gamma_shim_mpi_size(t));
  return 0;
}
static inline int MPI_Get_address(const void *p, MPI_Aint *a) { *a = (MPI_Aint)p; return 0; }
static inline int MPI_Type_create_struct(int n, const int *bl, const MPI_Aint *off,
                                         const MPI_Datatype *types, MPI_Datatype *out) {
  (void)n; (void)bl; (void)off; (void)types; *out = 100; return 0;
}
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }

static inline int gamma_shim_mpi_unreachable(const char *what) {
  fprintf(stderr, "oracle MPI shim: %s is unreachable with one rank\n", what);
  abort();
  return 1;
}
static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c;
  return gamma_shim_mpi_unreachable("MPI_Send");
}
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st;
  return gamma_shim_mpi_unreachable("MPI_Recv");
}
static inline int MPI_Sendrecv(const void *sb, int sn, MPI_Datatype st_, int d, int stag,
                               void *rb, int rn, MPI_Datatype rt, int s, int rtag,
                               MPI_Comm c, MPI_Status *st) {
  (void)sb; (void)sn; (void)st_; (void)d; (void)stag; (void)rb; (void)rn; (void)rt;
  (void)s; (void)rtag; (void)c; (void)st;
  return gamma_shim_mpi_unreachable("MPI_Sendrecv");
}

#endif
