/*
 * dropin_grid.c -- libgg_grid.so: the reference grid program's evaluator
 * interface (grid/common.h:88-90, grid/evaluation.c:192-209), served by the
 * B200 core library.  Link it where grid/Makefile links evaluation.o.
 *
 * Convention of grid/evaluation.c:182-189: false for a disconnected graph with
 * *diameter written (nodes+1) and *ASPL left untouched; true otherwise.  The
 * reference's queue BFS (enable_bfs) yields the same distance total and
 * diameter on a connected graph, so both settings use the GPU path.  The grid
 * program has no init hook, so the device is taken lazily on the first call.
 * Every other failure prints a message and aborts, as ERROR() does.
 */
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>

#define GGB_DROPIN_GRID
#include "../../include/graphgolf_b200.h"

extern void timer_start(const int n) __attribute__((weak));
extern void timer_stop(const int n) __attribute__((weak));

#define GGB_TIMER_APSP 2 /* grid/common.h:30 */

bool evaluation(const int nodes, const int degree, const int groups, const int *adjacency,
                const int based_nodes, const int height, const int based_height, int *diameter,
                double *ASPL, const bool enable_bfs, const int *rotate_hash)
{
  (void)height;
  (void)based_height;
  (void)enable_bfs;
  if (timer_start) timer_start(GGB_TIMER_APSP);
  ggb_result r;
  int rc = ggb_eval_grid(nodes, degree, groups, adjacency, based_nodes, rotate_hash, &r);
  if (rc) {
    fprintf(stdout, "graphgolf_b200: evaluation failed (%d): %s\n", rc, ggb_last_error());
    fflush(stdout);
    abort();
  }
  *diameter = r.diameter;
  if (r.connected) *ASPL = r.aspl;
  if (timer_stop) timer_stop(GGB_TIMER_APSP);
  return r.connected != 0;
}
