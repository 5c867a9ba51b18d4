/*
 * dropin_grid_nonregular.c -- libgg_grid_nr.so: the evaluator interface of the
 * reference's non-regular grid program
 * (variants/not_regular_grid_graph/common.h:86-88,
 * variants/not_regular_grid_graph/evaluation.c:192-207), served by the B200
 * core library.  Row i of adjacency holds degree[i] neighbours; conventions
 * and failure behaviour are those of libgg_grid.so.
 */
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>

#include "../../include/graphgolf_b200.h"

extern void timer_start(const int n) __attribute__((weak));
extern void timer_stop(const int n) __attribute__((weak));

#define GGB_TIMER_APSP 2 /* as grid/common.h:30 */

bool evaluation(const int nodes, const int max_degree, const int *degree, const int groups,
                const int *adjacency, const int based_nodes, const int height, const int based_height,
                int *diameter, double *ASPL, const bool enable_bfs, const int *rotate_hash)
{
  (void)height;
  (void)based_height;
  (void)enable_bfs;
  if (timer_start) timer_start(GGB_TIMER_APSP);
  ggb_result r;
  int rc = ggb_eval_grid_nonregular(nodes, max_degree, degree, groups, adjacency, based_nodes, rotate_hash, &r);
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
