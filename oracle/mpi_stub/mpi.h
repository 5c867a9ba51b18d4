/*
 * Single-process stand-in for <mpi.h>, used ONLY to compile the reference's
 * evaluator sources out-of-tree as a test oracle (oracle/_ref/).  There is no
 * MPI in this image.  Every call behaves as on a one-rank MPI_COMM_WORLD:
 * rank 0, size 1, and an in-place MPI_Allreduce leaves the buffer unchanged.
 */
#ifndef GGB_ORACLE_MPI_STUB_H
#define GGB_ORACLE_MPI_STUB_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_IN_PLACE ((void *)1)
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_C_BOOL 3
#define MPI_LONG_LONG 4
#define MPI_MAX 1
#define MPI_SUM 2
#define MPI_LAND 3
#define MPI_MAX_PROCESSOR_NAME 256

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Get_processor_name(char *name, int *len)
{
  strcpy(name, "localhost");
  *len = (int)strlen(name);
  return 0;
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c)
{
  (void)s; (void)r; (void)n; (void)t; (void)o; (void)c;  /* one rank: in place is the identity */
  return 0;
}
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; fflush(stdout); exit(code); }
#ifdef __cplusplus
}
#endif
#endif
