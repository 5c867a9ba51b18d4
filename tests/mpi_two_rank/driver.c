/*
 * Test driver (TEST INFRASTRUCTURE): an MPI host in the reference's shape --
 * the tentative `int rank, procs` of general/common.h:27, filled after
 * MPI_Init as general/main.c:330-332 does -- that evaluates one graph through
 * the drop-in evaluation() of libgg_general and prints its answer.
 * argv: adjacency file (int32, nodes*degree), nodes, based_nodes, groups,
 * degree, added_centers.
 */
#include <mpi.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>

int rank, procs;

bool evaluation(const int nodes, const int based_nodes, const int groups, const int lines, const int degree,
                int *adj, int *diameter, double *ASPL, const int added_centers, const int algo);
void init_matrix_dev(const int nodes, const int degree, const int based_nodes, const int algo);
void finalize_matrix_dev(void);

int main(int argc, char **argv)
{
  if (argc != 7) return 2;
  MPI_Init(&argc, &argv);
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  MPI_Comm_size(MPI_COMM_WORLD, &procs);
  const int nodes = atoi(argv[2]), based = atoi(argv[3]), groups = atoi(argv[4]), degree = atoi(argv[5]),
            ac = atoi(argv[6]);
  int *adj = malloc(sizeof(int) * (size_t)nodes * degree);
  FILE *f = fopen(argv[1], "rb");
  if (!f || fread(adj, sizeof(int), (size_t)nodes * degree, f) != (size_t)nodes * degree) return 2;
  fclose(f);
  init_matrix_dev(nodes, degree, based, 1);
  int diam = 0;
  double aspl = 0.0;
  const bool ok = evaluation(nodes, based, groups, nodes * degree / 2, degree, adj, &diam, &aspl, ac, 1);
  printf("%d %d %a\n", ok ? 1 : 0, diam, aspl);
  finalize_matrix_dev();
  free(adj);
  MPI_Finalize();
  return 0;
}
