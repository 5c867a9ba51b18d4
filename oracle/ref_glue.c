/*
 * ref_glue.c -- linked next to the reference's own evaluator sources when they
 * are compiled into oracle/_ref/ (test oracle only).  The reference keeps its
 * MPI rank and size in tentative globals (general/common.h:27,
 * grid/common.h:22) that main() normally fills (general/main.c:331-332); a
 * library has no main(), so the oracle sets them here.  procs > 1 with
 * rank 0 makes the reference evaluate only rank 0's share of the source
 * chunks (general/evaluation.c:166): a bounded sample of the same code path.
 */
extern int rank, procs;

void ref_set_ranks(int r, int p)
{
  rank = r;
  procs = p;
}

int ref_get_procs(void) { return procs; }
