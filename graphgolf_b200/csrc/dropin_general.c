/*
 * dropin_general.c -- libgg_general.so: the reference general program's
 * evaluator interface, served by the B200 core library.
 *
 * Link it where the reference links evaluation.o / evaluation_cuda.o
 * (general/Makefile:27-28,51-52).  It exports exactly the three symbols the
 * reference's host code calls:
 *   evaluation()          general/common.h:112-113, general/evaluation.cu:205-218
 *   init_matrix_dev()     general/main.c:3,420,   general/evaluation.cu:178-194
 *   finalize_matrix_dev() general/main.c:4,493,   general/evaluation.cu:196-203
 *
 * Return convention follows the CPU evaluator (general/evaluation.c:254-262):
 * true with the diameter and ASPL, or false with INT_MAX / DBL_MAX for a
 * disconnected graph.  Every other failure (CUDA error, adjacency entry out of
 * range, invalid sizes) prints a message and aborts the process, as the
 * reference's ERROR() does (general/common.h:67-70): returning false there
 * would make sa.c propose moves forever (general/sa.c:452-479).
 *
 * MPI hosts: built with -DGGB_WITH_MPI against the host's <mpi.h> (the
 * reference builds with mpicc, general/Makefile:1-8), a run with procs > 1
 * splits every evaluation as the reference's own evaluation() does: rank r
 * evaluates source windows r, r + procs, ... on its GPU (rank % gpus, as
 * init_matrix_dev picks it) and the ranks join diameter and distance sum with
 * two MPI_Allreduce calls (general/evaluation.c:166,247-248).  Without
 * -DGGB_WITH_MPI every rank evaluates the whole graph.
 */
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#ifdef GGB_WITH_MPI
#include <mpi.h>
#endif

#define GGB_DROPIN_GENERAL
#include "../../include/graphgolf_b200.h"

/* Supplied by the host program (general/timer.c, general/common.h:27).  Weak
 * so that the library also loads into a host that has neither. */
extern void timer_start(const int n) __attribute__((weak));
extern void timer_stop(const int n) __attribute__((weak));
extern int rank __attribute__((weak));
extern int procs __attribute__((weak));

#define GGB_TIMER_APSP 2 /* general/common.h:41 */

static void die(const char *what, int rc)
{
  fprintf(stdout, "graphgolf_b200: %s failed (%d): %s\n", what, rc, ggb_last_error());
  fflush(stdout);
  abort();
}

void init_matrix_dev(const int nodes, const int degree, const int based_nodes, const int algo)
{
  (void)based_nodes;
  (void)algo;
  /* general/evaluation.cu:181-184: GPU rank % gpus. */
  const int gpus = ggb_device_count();
  const int dev = (&rank != NULL && gpus > 0) ? rank % gpus : 0;
  int rc = ggb_init(gpus > 0 ? dev : -1, nodes, degree);
  if (rc) die("init_matrix_dev", rc);
}

void finalize_matrix_dev(void) { ggb_finalize(); }

bool evaluation(const int nodes, const int based_nodes, const int groups, const int lines,
                const int degree, int *adj, int *diameter, double *ASPL, const int added_centers,
                const int algo)
{
  (void)lines;
  (void)algo;
  if (timer_start) timer_start(GGB_TIMER_APSP);
  ggb_result r;
  int rc;
#ifdef GGB_WITH_MPI
  if (&procs != NULL && &rank != NULL && procs > 1) {
    ggb_partial p;
    rc = ggb_eval_general_partial(nodes, based_nodes, groups, degree, adj, added_centers, rank, procs, &p);
    if (rc) die("evaluation", rc);
    /* MAX of (diameter, disconnected, window width, -window width): every rank
     * must have cut the sources into the same windows */
    int mx[4] = {p.diam, p.disconnected, p.window_bits, -p.window_bits};
    long long sm = p.sum;
    MPI_Allreduce(MPI_IN_PLACE, mx, 4, MPI_INT, MPI_MAX, MPI_COMM_WORLD);
    MPI_Allreduce(MPI_IN_PLACE, &sm, 1, MPI_LONG_LONG, MPI_SUM, MPI_COMM_WORLD);
    if (mx[2] != -mx[3]) {
      fprintf(stdout, "graphgolf_b200: ranks cut the sources into different windows (%d and %d bits)\n", mx[2],
              -mx[3]);
      fflush(stdout);
      abort();
    }
    p.diam = mx[0];
    p.disconnected = mx[1];
    p.sum = sm;
    rc = ggb_finish_general(nodes, &p, &r);
  } else
#endif
  {
    rc = ggb_eval_general(nodes, based_nodes, groups, degree, adj, added_centers, &r);
  }
  if (rc) die("evaluation", rc);
  *diameter = r.diameter;
  *ASPL = r.aspl;
  if (timer_stop) timer_stop(GGB_TIMER_APSP);
  return r.connected != 0;
}
