/*
 * oracle/apsp_oracle.c -- CPU restatement of GraphGolf's exact APSP evaluator.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path in
 * graphgolf_b200/ is compared against.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may load it; the product never does.
 *
 * It restates, in plain C, the bit-parallel all-pairs BFS of the reference:
 *   - general/evaluation.c:153-263  matrix_op            (all sources, one pass per rank)
 *   - general/evaluation.c:265-373  matrix_op_mem_saving (4096-source passes, CHUNK=64 words)
 *   - general/evaluation.c:375-391  evaluation()          (dispatch, return convention)
 *   - grid/evaluation.c:122-190     matrix_op            (rotate_hash relabel, grid return convention)
 *   - variants/not_regular_general_graph/evaluation.c:156-393, variants/not_regular_grid_graph/
 *     evaluation.c:122-207: the same loops with a per-row neighbour count
 * and, as an independent second check, a plain queue BFS
 *   - general/evaluation.c:55-150   bfs (ASPL over half the matrix with symmetry weights)
 *
 * The reference accumulates the distance sum in a double that only ever holds
 * exact integers; here it is an int64 and is converted once, then divided by
 * the same double expression, which gives the identical double.
 *
 * Parity is pinned by comparing every function here with the reference's own
 * evaluator compiled from its sources (oracle/_ref, recipe in oracle/Makefile)
 * on the reference's data files and on seeded graphs (tests/test_oracle.py).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#include <float.h>

#define ORACLE_OK 0
#define ORACLE_EINVAL -1
#define ORACLE_ENOMEM -2

typedef struct {
  int nodes;           /* rows of the bitset matrices                      */
  int words;           /* uint64 words per row (the reference's `chunk`)   */
  int degree;
  const int *adj;      /* [nodes][degree]                                  */
  const int *relabel;  /* grid rotate_hash, or NULL for the identity       */
  const int *degs;     /* per-row neighbour counts (non-regular variants), or
                          NULL: every row has `degree` neighbours            */
} oracle_graph;

/* Per-level accounting of one source window: which rows the termination test
 * counts and how the unreached pairs are weighted into the sum.  The three
 * users are the general phase over the based sources, the general phase over
 * the added centres, and the grid. */
typedef struct {
  int split;          /* rows [0,split) are "lo", rows [split,nodes) are "hi"  */
  int term_hi_only;   /* 1: terminate when the hi rows are full (centre pass) */
  long long full_lo;  /* rows in lo that must be reached (per source)       */
  long long full_hi;
  long long w_lo;     /* weight of an unreached (lo row, source) pair       */
  long long w_hi;
} oracle_window_rule;

/* Runs one window of `l` sources whose identity bits sit in rows
 * first_row .. first_row+l-1 (bit i of row first_row+i), exactly as the
 * reference's level loop: B |= A[adj] (general/evaluation.c:175-181), count
 * (183-190), stop when full (192), swap (194-197), accumulate (199-200).
 * Returns the number of levels executed before the break, i.e. the loop
 * variable kk at exit (kk == nodes when the loop never broke). */
static long long run_window(const oracle_graph *g, uint64_t *A, uint64_t *B, int first_row, int l,
                            const oracle_window_rule *rule, long long *sum)
{
  const int n = g->nodes, w = g->words, d = g->degree;
  size_t cells = (size_t)n * (size_t)w;
  memset(A, 0, cells * sizeof(uint64_t));
  memset(B, 0, cells * sizeof(uint64_t));
  for (int i = 0; i < l; i++) {
    size_t off = (size_t)(first_row + i) * w + (size_t)(i / 64);
    A[off] = B[off] = 1ULL << (i % 64);
  }

  long long kk;
  for (kk = 0; kk < n; kk++) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      int row = g->relabel ? g->relabel[i] : i;
      uint64_t *dst = B + (size_t)row * w;
      /* non-regular variants: only the row's first degs[i] entries are edges
         (variants/not_regular_general_graph/evaluation.c:180, not_regular_grid_graph :149) */
      const int dj = g->degs ? g->degs[i] : d;
      for (int j = 0; j < dj; j++) {
        int nb = g->adj[(size_t)i * d + j];
        int src_row = g->relabel ? g->relabel[nb] : nb;
        const uint64_t *src = A + (size_t)src_row * w;
        for (int k = 0; k < w; k++) dst[k] |= src[k];
      }
    }
    unsigned long long lo = 0, hi = 0;
    size_t split_cells = (size_t)rule->split * w;
#pragma omp parallel for reduction(+ : lo) schedule(static)
    for (size_t c = 0; c < split_cells; c++) lo += (unsigned long long)__builtin_popcountll(B[c]);
#pragma omp parallel for reduction(+ : hi) schedule(static)
    for (size_t c = split_cells; c < cells; c++) hi += (unsigned long long)__builtin_popcountll(B[c]);

    int done = rule->term_hi_only ? (hi == (unsigned long long)(rule->full_hi * l))
                                  : (lo + hi == (unsigned long long)((rule->full_lo + rule->full_hi) * l));
    if (done) break;
    uint64_t *t = A; A = B; B = t;
    *sum += (rule->full_lo * l - (long long)lo) * rule->w_lo;
    *sum += (rule->full_hi * l - (long long)hi) * rule->w_hi;
  }
  return kk;
}

/*
 * Partial result of the general evaluator on one MPI rank, before the
 * MPI_Allreduce of general/evaluation.c:247-248.  words_per_row == 0 selects
 * MATRIX_OP's width (ceil(ceil(based_nodes/64)/procs), :157-158), any other
 * value a fixed width as MATRIX_OP_MEM_SAVING does with CHUNK=64 (:269-273).
 * Returns 0, or a negative error for invalid arguments / no memory.
 */
static int general_partial_impl(int nodes, int based_nodes, int groups, int degree, const int *adj,
                                const int *degs, int added_centers, int words_per_row, int rank, int procs,
                                int *diam_partial, long long *sum_partial)
{
  if (nodes <= 0 || based_nodes <= 0 || groups <= 0 || degree < 0 || procs <= 0 || rank < 0 ||
      rank >= procs || added_centers < 0 || based_nodes * groups + added_centers != nodes)
    return ORACLE_EINVAL;
  const int fixed = words_per_row > 0;
  unsigned elements = (unsigned)((based_nodes + 63) / 64);
  unsigned chunk = fixed ? (unsigned)words_per_row : (elements + procs - 1) / procs;
  unsigned parsize = (elements + chunk - 1) / chunk;
  unsigned alloc_words = chunk;
  if (added_centers && !fixed) {
    unsigned e2 = (unsigned)((added_centers + 63) / 64);
    unsigned c2 = (e2 + procs - 1) / procs;
    if (c2 > alloc_words) alloc_words = c2;  /* the reference reuses A/B; never larger in practice */
  }
  size_t cells = (size_t)nodes * alloc_words;
  uint64_t *A = malloc(cells * sizeof(uint64_t)), *B = malloc(cells * sizeof(uint64_t));
  if (!A || !B) { free(A); free(B); return ORACLE_ENOMEM; }

  oracle_graph g = {nodes, (int)chunk, degree, adj, NULL, degs};
  long long sum = 0;
  long long diam = 1;  /* *diam = 1 (:165) */

  /* Phase 1: the based sources (:166-203). */
  oracle_window_rule r1 = {based_nodes * groups, 0, (long long)based_nodes * groups, added_centers,
                           groups, 2LL * groups};
  for (unsigned t = (unsigned)rank; t < parsize; t += procs) {
    long long first = 64LL * t * chunk;
    int l = (int)((based_nodes - first) < 64LL * chunk ? (based_nodes - first) : 64LL * chunk);
    long long kk = run_window(&g, A, B, (int)first, l, &r1, &sum);
    if (kk + 1 > diam) diam = kk + 1;
  }

  /* Phase 2: the added centres (:205-245). */
  if (added_centers) {
    unsigned e2 = (unsigned)((added_centers + 63) / 64);
    unsigned c2 = fixed ? chunk : (e2 + procs - 1) / procs;
    unsigned p2 = (e2 + c2 - 1) / c2;
    int s = based_nodes % procs;
    int new_rank = (rank - s >= 0) ? rank - s : rank - s + procs;
    /* the non-regular variant's centre phase reads whole rows
     * (variants/not_regular_general_graph/evaluation.c:226) */
    oracle_graph g2 = {nodes, (int)c2, degree, adj, NULL, NULL};
    oracle_window_rule r2 = {based_nodes * groups, 1, 0, added_centers, 0, 1};
    for (unsigned t = (unsigned)new_rank; t < p2; t += procs) {
      long long first = 64LL * t * c2;
      int l = (int)((added_centers - first) < 64LL * c2 ? (added_centers - first) : 64LL * c2);
      long long kk = run_window(&g2, A, B, (int)(first + nodes - added_centers), l, &r2, &sum);
      if (kk + 1 > diam) diam = kk + 1;
    }
  }
  free(A);
  free(B);
  *diam_partial = diam > INT_MAX ? INT_MAX : (int)diam;
  *sum_partial = sum;
  return ORACLE_OK;
}

int oracle_general_partial(int nodes, int based_nodes, int groups, int degree, const int *adj,
                           int added_centers, int words_per_row, int rank, int procs,
                           int *diam_partial, long long *sum_partial)
{
  return general_partial_impl(nodes, based_nodes, groups, degree, adj, NULL, added_centers, words_per_row, rank,
                              procs, diam_partial, sum_partial);
}

/* The tail of general/evaluation.c:247-262 once the partials are reduced
 * (MAX of diameters, SUM of sums): add N(N-1), divide, or report a
 * disconnected graph as diameter INT_MAX and ASPL DBL_MAX. */
int oracle_general_finish(int nodes, int diam, long long sum, int *diameter, double *ASPL)
{
  double total = (double)(sum + (long long)nodes * (nodes - 1));
  if (diam < nodes) {
    *diameter = diam;
    *ASPL = total / (((double)nodes - 1) * nodes);
    return 1;
  }
  *diameter = INT_MAX;
  *ASPL = DBL_MAX;
  return 0;
}

/* general evaluation() with algo MATRIX_OP (1) or MATRIX_OP_MEM_SAVING (2) on
 * one rank.  Returns 1 (connected), 0 (disconnected) or a negative error.
 * *sum_out receives the exact integer the reference divides (sum + N(N-1)). */
int oracle_general_eval(int nodes, int based_nodes, int groups, int degree, const int *adj,
                        int added_centers, int algo, int *diameter, double *ASPL, long long *sum_out)
{
  int dp;
  long long sp;
  int rc = oracle_general_partial(nodes, based_nodes, groups, degree, adj, added_centers,
                                  algo == 2 ? 64 : 0, 0, 1, &dp, &sp);
  if (rc) return rc;
  if (sum_out) *sum_out = sp + (long long)nodes * (nodes - 1);
  return oracle_general_finish(nodes, dp, sp, diameter, ASPL);
}

/* variants/not_regular_general_graph/evaluation.c:156-393: the same with
 * row i holding num_degrees[i] neighbours (max_degree slots). */
int oracle_general_eval_nr(int nodes, int based_nodes, int groups, int max_degree, const int *num_degrees,
                           const int *adj, int added_centers, int algo, int *diameter, double *ASPL,
                           long long *sum_out)
{
  int dp;
  long long sp;
  int rc = general_partial_impl(nodes, based_nodes, groups, max_degree, adj, num_degrees, added_centers,
                                algo == 2 ? 64 : 0, 0, 1, &dp, &sp);
  if (rc) return rc;
  if (sum_out) *sum_out = sp + (long long)nodes * (nodes - 1);
  return oracle_general_finish(nodes, dp, sp, diameter, ASPL);
}

/* grid/evaluation.c:122-190 on one rank: the same level loop over relabelled
 * rows, sources = relabelled ids 0..based_nodes-1, weight `groups`.  The grid
 * convention differs from the general one: disconnected means diameter >
 * nodes, the diameter is still written, and ASPL is left untouched. */
static int grid_partial_impl(int nodes, int degree, const int *degs, int groups, const int *adj, int based_nodes,
                             const int *rotate_hash, int rank, int procs, int *diam_partial, long long *sum_partial)
{
  if (nodes <= 0 || based_nodes <= 0 || groups <= 0 || degree < 0 || procs <= 0 || rank < 0 || rank >= procs)
    return ORACLE_EINVAL;
  unsigned elements = (unsigned)((based_nodes + 63) / 64);
  unsigned chunk = (elements + procs - 1) / procs;
  unsigned parsize = (elements + chunk - 1) / chunk;
  size_t cells = (size_t)nodes * chunk;
  uint64_t *A = malloc(cells * sizeof(uint64_t)), *B = malloc(cells * sizeof(uint64_t));
  if (!A || !B) { free(A); free(B); return ORACLE_ENOMEM; }
  oracle_graph g = {nodes, (int)chunk, degree, adj, rotate_hash, degs};
  oracle_window_rule r = {nodes, 0, nodes, 0, groups, 0};
  long long sum = 0, diam = 1;
  for (unsigned t = (unsigned)rank; t < parsize; t += procs) {
    long long first = 64LL * t * chunk;
    int l = (int)((based_nodes - first) < 64LL * chunk ? (based_nodes - first) : 64LL * chunk);
    long long kk = run_window(&g, A, B, (int)first, l, &r, &sum);
    if (kk + 1 > diam) diam = kk + 1;
  }
  free(A);
  free(B);
  *diam_partial = diam > INT_MAX ? INT_MAX : (int)diam;
  *sum_partial = sum;
  return ORACLE_OK;
}

int oracle_grid_partial(int nodes, int degree, int groups, const int *adj, int based_nodes,
                        const int *rotate_hash, int rank, int procs, int *diam_partial, long long *sum_partial)
{
  return grid_partial_impl(nodes, degree, NULL, groups, adj, based_nodes, rotate_hash, rank, procs, diam_partial,
                           sum_partial);
}

int oracle_grid_finish(int nodes, int diam, long long sum, int *diameter, double *ASPL)
{
  double total = (double)(sum + (long long)nodes * (nodes - 1));
  *diameter = diam;
  if (diam > nodes) return 0;
  *ASPL = total / (((double)nodes - 1) * nodes);
  return 1;
}

int oracle_grid_eval(int nodes, int degree, int groups, const int *adj, int based_nodes,
                     const int *rotate_hash, int *diameter, double *ASPL, long long *sum_out)
{
  int dp;
  long long sp;
  int rc = oracle_grid_partial(nodes, degree, groups, adj, based_nodes, rotate_hash, 0, 1, &dp, &sp);
  if (rc) return rc;
  if (sum_out) *sum_out = sp + (long long)nodes * (nodes - 1);
  return oracle_grid_finish(nodes, dp, sp, diameter, ASPL);
}

/*
 * Independent check: plain queue BFS from every source s < n_sources over the
 * (optionally relabelled) graph.  Returns the largest eccentricity and the
 * sum over sources of the distances to every vertex, or -1 in *ecc_max when
 * some vertex is unreachable.  Weighting by `groups` and the N(N-1) term are
 * left to the caller; this only follows the definition of distance, not any
 * reference code, so it catches a shared misreading of the bitset recurrence.
 */
int oracle_bfs_sums(int nodes, int degree, const int *adj, const int *relabel, int n_sources,
                    int *ecc_max, long long *dist_sum)
{
  int *dist = malloc(sizeof(int) * nodes), *queue = malloc(sizeof(int) * nodes);
  int *inv = relabel ? malloc(sizeof(int) * nodes) : NULL;
  if (!dist || !queue || (relabel && !inv)) { free(dist); free(queue); free(inv); return ORACLE_ENOMEM; }
  if (relabel) for (int i = 0; i < nodes; i++) inv[relabel[i]] = i;
  long long total = 0;
  int emax = 0;
  for (int s = 0; s < n_sources; s++) {
    int s_orig = relabel ? inv[s] : s;
    for (int i = 0; i < nodes; i++) dist[i] = -1;
    int head = 0, tail = 0;
    dist[s_orig] = 0;
    queue[tail++] = s_orig;
    while (head < tail) {
      int v = queue[head++];
      for (int j = 0; j < degree; j++) {
        int u = adj[(size_t)v * degree + j];
        if (dist[u] < 0) { dist[u] = dist[v] + 1; queue[tail++] = u; }
      }
    }
    if (tail != nodes) { emax = -1; break; }
    for (int i = 0; i < nodes; i++) {
      total += dist[i];
      if (dist[i] > emax) emax = dist[i];
    }
  }
  free(dist);
  free(queue);
  free(inv);
  *ecc_max = emax;
  *dist_sum = total;
  return ORACLE_OK;
}

/* variants/not_regular_grid_graph/evaluation.c:122-190: the grid level loop
 * with row i holding degree[i] neighbours (max_degree slots). */
int oracle_grid_eval_nr(int nodes, int max_degree, const int *degree, int groups, const int *adj, int based_nodes,
                        const int *rotate_hash, int *diameter, double *ASPL, long long *sum_out)
{
  int dp;
  long long sp;
  int rc = grid_partial_impl(nodes, max_degree, degree, groups, adj, based_nodes, rotate_hash, 0, 1, &dp, &sp);
  if (rc) return rc;
  if (sum_out) *sum_out = sp + (long long)nodes * (nodes - 1);
  return oracle_grid_finish(nodes, dp, sp, diameter, ASPL);
}
