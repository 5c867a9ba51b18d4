/*
 * dropin_general_nonregular.c -- libgg_general_nr.so: the evaluator interface
 * of the reference's non-regular general program
 * (variants/not_regular_general_graph/common.h:103-105,
 * variants/not_regular_general_graph/evaluation.c:378-393), served by the
 * B200 core library.  Link it where that program's Makefile links
 * evaluation.o.  Row i of adj holds num_degrees[i] neighbours; conventions and
 * failure behaviour are those of libgg_general.so.  The program has no init
 * hook: the device is taken on the first call.
 */
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>

#include "../../include/graphgolf_b200.h"

extern void timer_start(const int n) __attribute__((weak));
extern void timer_stop(const int n) __attribute__((weak));

#define GGB_TIMER_APSP 2 /* variants/not_regular_general_graph/common.h, as general/common.h:41 */

bool evaluation(const int nodes, const int based_nodes, const int groups, const int lines, const int degree,
                int *adj, int *diameter, double *ASPL, const int added_centers, const int *num_degrees,
                const int algo)
{
  (void)lines;
  (void)algo;
  if (timer_start) timer_start(GGB_TIMER_APSP);
  ggb_result r;
  int rc = ggb_eval_general_nonregular(nodes, based_nodes, groups, degree, num_degrees, adj, added_centers, &r);
  if (rc) {
    fprintf(stdout, "graphgolf_b200: evaluation failed (%d): %s\n", rc, ggb_last_error());
    fflush(stdout);
    abort();
  }
  *diameter = r.diameter;
  *ASPL = r.aspl;
  if (timer_stop) timer_stop(GGB_TIMER_APSP);
  return r.connected != 0;
}
