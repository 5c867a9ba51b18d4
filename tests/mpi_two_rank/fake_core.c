/*
 * CPU stand-in for the core library's entry points that libgg_general calls
 * (TEST INFRASTRUCTURE): the per-rank partial comes from the oracle's C
 * restatement of the reference's evaluator (oracle/apsp_oracle.c) over
 * 128-source windows, so the shim's rank split and all-reduce can be tested
 * without a GPU.  Declarations as in include/graphgolf_b200.h.
 */
#include <float.h>
#include <limits.h>
#include <stddef.h>

#include "../../include/graphgolf_b200.h"

int oracle_general_partial(int nodes, int based_nodes, int groups, int degree, const int *adj, int added_centers,
                           int words_per_row, int rank, int procs, int *diam_partial, long long *sum_partial);

int ggb_init(int device, int nodes, int degree) { (void)device; (void)nodes; (void)degree; return GGB_OK; }
void ggb_finalize(void) {}
int ggb_device_count(void) { return 1; }
const char *ggb_last_error(void) { return "fake core"; }

int ggb_eval_general_partial(int nodes, int based_nodes, int groups, int degree, const int *adj, int added_centers,
                             int rank, int procs, ggb_partial *out)
{
  int diam = 0;
  long long sum = 0;
  if (oracle_general_partial(nodes, based_nodes, groups, degree, adj, added_centers, 2, rank, procs, &diam, &sum))
    return GGB_EINVAL;
  out->diam = diam;
  out->disconnected = diam >= nodes;
  out->sum = sum;
  out->levels = 0;
  out->windows = 0;
  out->window_bits = 128;
  out->dense_levels = 0;
  return GGB_OK;
}

int ggb_finish_general(int nodes, const ggb_partial *p, ggb_result *out)
{
  if (!p->disconnected && p->diam < nodes) {
    out->connected = 1;
    out->diameter = p->diam;
    out->total = p->sum + (long long)nodes * (nodes - 1);
    out->aspl = (double)out->total / (((double)nodes - 1) * nodes);
  } else {
    out->connected = 0;
    out->diameter = INT_MAX;
    out->aspl = DBL_MAX;
    out->total = 0;
  }
  return GGB_OK;
}

int ggb_eval_general(int nodes, int based_nodes, int groups, int degree, const int *adj, int added_centers,
                     ggb_result *out)
{
  ggb_partial p;
  int rc = ggb_eval_general_partial(nodes, based_nodes, groups, degree, adj, added_centers, 0, 1, &p);
  return rc ? rc : ggb_finish_general(nodes, &p, out);
}
