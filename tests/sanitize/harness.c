/*
 * Sanitizer harness (TEST INFRASTRUCTURE): drives the host C code of the
 * package (graphgolf_b200/csrc/host/graph_host.c) and the oracle's C
 * restatement (oracle/apsp_oracle.c) through their entry points, built with
 * -fsanitize=address,undefined, so that an out-of-bounds access, a leak or
 * undefined behaviour on these paths fails the test.  argv[1]: a scratch
 * directory for the edge files.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int ggbh_random_regular(int n, int d, uint64_t seed, int *edges);
int ggbh_symmetric_regular(int n, int d, int g, uint64_t seed, int *edges);
int ggbh_grid_regular(int W, int H, int d, int R, long long swaps, uint64_t seed, int *edges);
int ggbh_create_adj(int n, int lines, int d, const int *edges, int *adj);
int ggbh_rotate_hash(int n, int height, int width, int groups, int *rh);
long long ggbh_count_lines(const char *path);
long long ggbh_read_general(const char *path, int *edges, long long max_lines);
int ggbh_write_general(const char *path, long long lines, const int *edges);
long long ggbh_read_grid(const char *path, int *edges, long long max_lines, int *width, int *height);
int ggbh_write_grid(const char *path, long long lines, const int *edges, int height);
int ggbh_verify(int n, long long lines, int d, const int *edges, int max_len, int height);
int oracle_general_eval(int nodes, int based_nodes, int groups, int degree, const int *adj, int added_centers,
                        int algo, int *diameter, double *ASPL, long long *sum_out);
int oracle_grid_eval(int nodes, int degree, int groups, const int *adj, int based_nodes, const int *rotate_hash,
                     int *diameter, double *ASPL, long long *sum_out);
int oracle_bfs_sums(int nodes, int degree, const int *adj, const int *relabel, int n_sources, int *ecc,
                    long long *sum);

#define CHECK(c)                                                     \
  do {                                                               \
    if (!(c)) {                                                      \
      fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
      return 1;                                                      \
    }                                                                \
  } while (0)

static int general_case(const char *dir, int n, int d, int g, uint64_t seed)
{
  const int lines = n * d / 2;
  int *e = malloc(sizeof(int) * 2 * lines), *e2 = malloc(sizeof(int) * 2 * lines);
  int *adj = malloc(sizeof(int) * n * d);
  CHECK((g > 1 ? ggbh_symmetric_regular(n, d, g, seed, e) : ggbh_random_regular(n, d, seed, e)) == 0);
  CHECK(ggbh_verify(n, lines, d, e, 0, 0) == 0);
  CHECK(ggbh_create_adj(n, lines, d, e, adj) == 0);
  char path[1024];
  snprintf(path, sizeof path, "%s/g_%d_%d_%d.edges", dir, n, d, g);
  CHECK(ggbh_write_general(path, lines, e) == 0);
  CHECK(ggbh_count_lines(path) == lines);
  CHECK(ggbh_read_general(path, e2, lines) == lines);
  CHECK(memcmp(e, e2, sizeof(int) * 2 * lines) == 0);
  int diam = 0, ecc = 0;
  double aspl = 0.0;
  long long sum = 0, bsum = 0;
  CHECK(oracle_general_eval(n, n / g, g, d, adj, 0, 1, &diam, &aspl, &sum) == 1);
  int diam2 = 0;
  double aspl2 = 0.0;
  long long sum2 = 0;
  CHECK(oracle_general_eval(n, n / g, g, d, adj, 0, 2, &diam2, &aspl2, &sum2) == 1);
  CHECK(diam == diam2 && sum == sum2);
  if (g == 1) {
    CHECK(oracle_bfs_sums(n, d, adj, NULL, n, &ecc, &bsum) == 0);
    CHECK(ecc == diam && bsum == sum);   /* queue BFS: the same distance total */
  }
  /* an invalid edge list is rejected, not read out of bounds */
  e[0] = n + 5;
  CHECK(ggbh_create_adj(n, lines, d, e, adj) != 0);
  CHECK(ggbh_verify(n, lines, d, e, 0, 0) != 0);
  free(e);
  free(e2);
  free(adj);
  return 0;
}

static int grid_case(const char *dir, int w, int h, int d, int r, int g, uint64_t seed)
{
  const int n = w * h, lines = n * d / 2;
  int *e = malloc(sizeof(int) * 2 * lines), *e2 = malloc(sizeof(int) * 2 * lines);
  int *adj = malloc(sizeof(int) * n * d), *rh = malloc(sizeof(int) * n);
  CHECK(ggbh_grid_regular(w, h, d, r, 20LL * lines, seed, e) == 0);
  CHECK(ggbh_verify(n, lines, d, e, r, h) == 0);
  CHECK(ggbh_create_adj(n, lines, d, e, adj) == 0);
  CHECK(ggbh_rotate_hash(n, h, w, g, rh) == 0);
  char path[1024];
  snprintf(path, sizeof path, "%s/w%dh%d.edges", dir, w, h);
  CHECK(ggbh_write_grid(path, lines, e, h) == 0);
  int ww = 0, hh = 0;
  CHECK(ggbh_read_grid(path, e2, lines, &ww, &hh) == lines);
  CHECK(ww == w && hh == h);
  int diam = 0;
  double aspl = 0.0;
  long long sum = 0;
  CHECK(oracle_grid_eval(n, d, g, adj, n / g, rh, &diam, &aspl, &sum) >= 0);
  free(e);
  free(e2);
  free(adj);
  free(rh);
  return 0;
}

int main(int argc, char **argv)
{
  if (argc < 2) return 2;
  int rc = 0;
  rc |= general_case(argv[1], 64, 3, 1, 1);
  rc |= general_case(argv[1], 500, 6, 1, 2);
  rc |= general_case(argv[1], 512, 8, 4, 3);
  rc |= general_case(argv[1], 1000, 5, 1, 4);
  rc |= grid_case(argv[1], 10, 10, 4, 3, 1, 5);
  rc |= grid_case(argv[1], 20, 20, 6, 3, 2, 6);
  rc |= grid_case(argv[1], 16, 16, 4, 2, 4, 7);
  if (!rc) printf("sanitized host and oracle paths: ok\n");
  return rc;
}
