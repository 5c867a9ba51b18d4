/*
 * graphgolf_b200.h -- C ABI of the B200 exact APSP evaluator.
 *
 * Two layers are declared here.
 *
 * 1. The core library  (graphgolf_b200/_lib/libgraphgolf_b200.so), prefix ggb_.
 *    Plain pointers and sizes; no CUDA or torch types in any signature.  A
 *    stream is passed as `void *` (a cudaStream_t, or NULL for the library's
 *    own stream).
 *
 * 2. The drop-in shims that replace the reference's evaluator at link time:
 *    libgg_general.so exports the general evaluation()/init_matrix_dev()/
 *    finalize_matrix_dev() and libgg_grid.so exports the grid evaluation().
 *    They carry the reference's names and signatures, so they are declared in
 *    two guarded blocks below (the two evaluation() signatures clash and can
 *    never be in one translation unit, exactly as in the reference).
 *
 * Numerical contract: the diameter and the integer distance total are
 * bit-exact against the reference's CPU evaluator (general/evaluation.c,
 * grid/evaluation.c), and ASPL is the same double, computed by the same
 * expression from the same integer.
 */
#ifndef GRAPHGOLF_B200_H
#define GRAPHGOLF_B200_H

#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes returned by every ggb_ function ---------------------- */
#define GGB_OK 0
#define GGB_EINVAL -1    /* argument out of the supported domain            */
#define GGB_ECUDA -2     /* a CUDA runtime call failed                       */
#define GGB_EADJ -3      /* an adjacency entry is outside [0, nodes)         */
#define GGB_ETIMEOUT -4  /* a bounded device-side wait ran out               */
#define GGB_EPERM -5     /* rotate_hash is not a permutation of [0, nodes)   */
#define GGB_ENOMEM -6    /* device or pinned host memory could not be had    */

/* Result of one evaluation.  `connected` is the reference evaluation()'s
 * return value; `diameter` and `aspl` are what it writes through its
 * pointers (see ggb_eval_general / ggb_eval_grid for the two conventions). */
typedef struct ggb_result {
  int connected;        /* 1: every pair reached; 0: disconnected              */
  int diameter;         /* general: INT_MAX if disconnected; grid: nodes+1     */
  double aspl;          /* general: DBL_MAX if disconnected; grid: NaN (the
                           reference leaves its ASPL untouched in that case)  */
  long long total;      /* exact Σ over ordered pairs of d(u,v), weighted by
                           the symmetry groups = the reference's `sum` after
                           `sum += nodes*(nodes-1)`; 0 if disconnected        */
  long long levels;     /* BFS levels executed, summed over source windows   */
  int windows;          /* source windows run                                 */
  int window_bits;      /* sources per window (64 or a multiple of 128)       */
  long long dense_levels; /* of `levels`, those run as dense OR-gather sweeps
                           (the first two levels of a window are seeded from
                           the two-hop adjacency instead)                     */
} ggb_result;

/* Partial result of a rank that ran a strided share of the source windows
 * (the reference's MPI decomposition, general/evaluation.c:166).  Combine
 * partials with MAX on `diam` and SUM on `sum`, then ggb_finish_*(). */
typedef struct ggb_partial {
  int diam;             /* max over this rank's windows of levels-to-full (1 if none) */
  int disconnected;     /* 1 if a window of this rank found an unreachable pair       */
  long long sum;        /* Σ weighted unreached (vertex, source) pairs per level      */
  long long levels;
  int windows;
  int window_bits;
  long long dense_levels;
} ggb_partial;

/* ---- lifecycle --------------------------------------------------------- */

/* Selects the device for this thread and creates the library's stream and
 * grow-only buffers for graphs up to `nodes` x `degree` (0, 0 = lazily).
 * Replaces init_matrix_dev (general/evaluation.cu:178-194). */
int ggb_init(int device, int nodes, int degree);

/* Frees every device and pinned buffer.  Replaces finalize_matrix_dev
 * (general/evaluation.cu:196-203).  Safe to call twice. */
void ggb_finalize(void);

/* Text of the last error on this process ("" if none). */
const char *ggb_last_error(void);

/* Library version string. */
const char *ggb_version(void);

/* Number of CUDA devices visible to this process (0 if none or on error). */
int ggb_device_count(void);

/* Forces the source-window width (bits: 64, or 128 * 2^k up to 8192; 0 =
 * automatic) and the persistent grid size (CTAs, 0 = automatic).  Used by the
 * autotuner and by tests and benchmarks that sweep widths; results never
 * depend on either.  64-source windows (the reference's one-word chunk,
 * general/evaluation.cu:27-44) keep one 16-byte row per vertex with its upper
 * half zero: a gather fetches one 32-byte L2 sector either way. */
int ggb_set_tuning(int window_bits, int ctas);

/* Policy for the ball pre-pass (one kernel that writes S_3 of every source
 * window, so that windows start their dense sweeps at level 3): -1 automatic
 * by the cost model, 0 never, 1 whenever the sizes allow it (degree <= 32,
 * at most 64 windows per rank, the row fits in shared memory).  Results
 * never depend on it. */
int ggb_set_ball(int mode);

/* Test hook for the bounded device waits: every grid-barrier wait gives up
 * after timeout_ns, and `phantom` extra arrivals that never come are added to
 * every barrier.  phantom=1 makes each wait run out, which must surface as
 * GGB_ETIMEOUT with the CUDA context still usable.  (2e9, 0) restores the
 * default. */
int ggb_set_barrier_test(long long timeout_ns, int phantom);

/* Opt-in timeline of the persistent kernel: with capacity > 0, CTA 0 records
 * a (globaltimer ns, tag | level << 8) pair after every grid barrier of the
 * following evaluations (tag 1: a window's two seeded levels, tag 2: a dense
 * sweep).  0 turns it off.  The device-side analogue of the reference's
 * TIMER_APSP bracket (general/timer.c), one level finer. */
int ggb_trace_enable(int capacity);

/* Copies the last evaluation's trace pairs to out (2*max_pairs long longs);
 * returns the number of pairs copied. */
int ggb_trace_read(long long *out, int max_pairs);

/* Per-kernel timing: with enable != 0, CUDA events are recorded on the
 * launching stream around the ball pre-pass and the persistent kernel of
 * every following evaluation; ggb_kernel_times returns the last one's
 * milliseconds (ball 0 when it did not run).  No counterpart in the
 * reference; bench.py's roofline uses it. */
int ggb_set_timing(int enable);
int ggb_kernel_times(double *ms_ball, double *ms_persistent);

/* The dense sweeps' own access pattern as a probe: random-row OR sweeps (d
 * random neighbours per row, rows of window_bits/8 bytes, N rows) with the
 * sweeps' access width (32-byte loads for rows of 32 bytes or more), one
 * launch per sweep, on the current device with its own buffers.  *gbs counts
 * the algorithmic bytes of a dense sweep (N*d*4 + N*d*W/8 + 2*N*W/8) per
 * second; bench.py reports it beside the roofline's peak.  No counterpart
 * in the reference; a measurement utility for the roofline. */
int ggb_probe_l2_gather(int N, int d, int window_bits, int iters, double *gbs);

/* The L2 streaming ceiling, the roofline's peak in bench.py: GB/s at which an
 * L2-resident buffer of `mib` MiB (1..96) reaches the SMs' shared memory
 * through bulk copies, one CTA per SM with about 192 KB in flight, averaged
 * over `iters` launches.  No counterpart in the reference; a measurement
 * utility for the roofline. */
int ggb_probe_l2_stream(int mib, int iters, double *gbs);

/* ---- host-buffer entry points (copy in, evaluate, copy out) ------------ */

/* General graph: replaces evaluation() of general/evaluation.c:375-391 with
 * algo MATRIX_OP / MATRIX_OP_MEM_SAVING (general/common.h:59-60), including
 * added centres (-v).  adj is the caller's [nodes][degree] int32 array; it
 * is read during the call only.  nodes must equal based_nodes*groups +
 * added_centers (general/main.c:375-382).  Disconnected: connected=0,
 * diameter=INT_MAX, aspl=DBL_MAX (general/evaluation.c:254-262). */
int ggb_eval_general(int nodes, int based_nodes, int groups, int degree, const int *adj,
                     int added_centers, ggb_result *out);

/* Grid graph: replaces evaluation() of grid/evaluation.c:192-209 (matrix
 * path).  rotate_hash is create_rotate_hash's relabel (grid/common.c:312-341)
 * and must be a permutation.  Disconnected: connected=0, diameter=nodes+1 as
 * the reference writes it, aspl=NaN (the reference leaves it untouched). */
int ggb_eval_grid(int nodes, int degree, int groups, const int *adj, int based_nodes,
                  const int *rotate_hash, ggb_result *out);

/* Non-regular general graph: replaces evaluation() of
 * variants/not_regular_general_graph/evaluation.c:378-393.  Row i of the
 * [nodes][max_degree] adjacency holds num_degrees[i] neighbours; the BFS over
 * the based sources reads only those (:180), the added-centre phase reads the
 * whole row, padding included, as the reference does (:226).  Same return
 * convention as ggb_eval_general; num_degrees[i] outside [0, max_degree] is
 * rejected with GGB_EINVAL. */
int ggb_eval_general_nonregular(int nodes, int based_nodes, int groups, int max_degree, const int *num_degrees,
                                const int *adj, int added_centers, ggb_result *out);

/* Non-regular grid graph: replaces evaluation() of
 * variants/not_regular_grid_graph/evaluation.c:192-207 (matrix path); row i
 * holds degree[i] neighbours (:149-151).  Grid return convention. */
int ggb_eval_grid_nonregular(int nodes, int max_degree, const int *degree, int groups, const int *adj,
                             int based_nodes, const int *rotate_hash, ggb_result *out);

/* ---- device-resident entry points (inputs already in HBM) -------------- */

/* Same as ggb_eval_general with adj_dev a device pointer.  Enqueues on
 * `stream` and waits for the result. */
int ggb_eval_general_device(int nodes, int based_nodes, int groups, int degree, const int *adj_dev,
                            int added_centers, void *stream, ggb_result *out);

/* Enqueues one general evaluation on `stream` without waiting: the result
 * stays on the device until ggb_collect() on the same stream.  Used to time
 * back-to-back evaluations with events on the launching stream. */
int ggb_launch_general_device(int nodes, int based_nodes, int groups, int degree, const int *adj_dev,
                              int added_centers, void *stream);

/* Waits for the last launch on `stream` and returns its result. */
int ggb_collect(void *stream, ggb_result *out);

/* Number of this library's kernels enqueued since load: every kernel of an
 * evaluation (ball pre-pass, persistent kernel, the grid relabel kernels, the
 * widening of 16-bit ids after an upload) counts once per launch. */
long long ggb_kernel_launches(void);

/* Bytes of adjacency this library has copied from host to device since load:
 * what the host-buffer entry points send over PCIe (2 bytes per id when the
 * ids fit 16 bits, else 4). */
long long ggb_h2d_bytes(void);

/* ---- evaluation without device allocation ------------------------------- */

/* No counterpart in the reference.  For callers that cannot let a library
 * call cudaMalloc -- a host whose device memory belongs to another allocator
 * (a framework's caching pool, a fixed budget carved out at start-up) or an
 * annealing loop that must not allocate while it runs.  Same result as
 * ggb_eval_general_device; allocates nothing: the kernel's scratch lives in a
 * 16 MiB file-scope device array (ggb_noalloc_scratch_bytes()) that every GPU
 * loading this library holds until exit, so nodes must be at most 524280
 * (larger graphs are rejected with GGB_EINVAL).  adj_dev is a device pointer,
 * `out` a host pointer; the call waits for its result on `stream` (NULL: the
 * default stream).  The first call on a device looks up the array's device
 * address; make it before any stream capture.  All calls share the one array:
 * calls that overlap on the GPU (two threads or two streams) race and must be
 * serialised by the caller. */
int ggb_eval_general_noalloc(int nodes, int based_nodes, int groups, int degree, const int *adj_dev,
                             int added_centers, void *stream, ggb_result *out);

/* Size in bytes of the device array ggb_eval_general_noalloc works in. */
long long ggb_noalloc_scratch_bytes(void);

/* Text of the last error of ggb_eval_general_noalloc ("" if none). */
const char *ggb_noalloc_last_error(void);

/* ---- multi-rank decomposition (one GPU per rank) ------------------------ */

/* Runs only the source windows t = rank, rank+procs, ... of a general graph
 * (the reference's MPI split, general/evaluation.c:166,212) on this process's
 * GPU and returns the partial.  Host buffer in, partial out. */
int ggb_eval_general_partial(int nodes, int based_nodes, int groups, int degree, const int *adj,
                             int added_centers, int rank, int procs, ggb_partial *out);

/* Device-resident form of ggb_eval_general_partial: enqueues rank's share
 * on `stream` without waiting; ggb_collect_partial waits and returns it.
 * Used to time the sharded evaluation (bench.py --shard). */
int ggb_launch_general_partial_device(int nodes, int based_nodes, int groups, int degree, const int *adj_dev,
                                      int added_centers, int rank, int procs, void *stream);
int ggb_collect_partial(void *stream, ggb_partial *out);

/* Completes reduced partials into the general convention
 * (general/evaluation.c:247-262). */
int ggb_finish_general(int nodes, const ggb_partial *reduced, ggb_result *out);

/* Completes reduced partials into the grid convention
 * (grid/evaluation.c:176-189). */
int ggb_finish_grid(int nodes, const ggb_partial *reduced, ggb_result *out);

/* ---- batches: many graphs, of uneven sizes, in one launch --------------- */

/* A batch is a fixed list of general graphs (ac = 0) whose adjacency arrays
 * live packed in one device buffer; one cooperative launch, captured once in a
 * CUDA graph and replayed, evaluates them all.  Its CTAs form teams of
 * team_ctas CTAs; the graphs are dealt to the teams longest-first; every team
 * runs its graphs' source windows of window_bits sources with a barrier of its
 * own.  Each graph's result is the one ggb_eval_general gives it
 * (general/evaluation.c:153-263 per graph, :249-262 for the convention).  No
 * counterpart in the reference, whose evaluation() takes one graph.
 * A batch belongs to the device current at ggb_batch_create; it is not
 * thread-safe. */
typedef struct ggb_batch ggb_batch;

/* Creates a batch of n_graphs graphs; graph i has nodes[i] vertices,
 * based_nodes[i] * groups[i] == nodes[i], degree[i] neighbours per row.  The
 * initial plan is the cost model's choice. */
int ggb_batch_create(int n_graphs, const int *nodes, const int *based_nodes, const int *groups,
                     const int *degree, ggb_batch **out);
void ggb_batch_destroy(ggb_batch *b);

/* Fixes the plan: window_bits = 128 * 2^k (<= 4096), team_ctas >= 1; a 0
 * leaves that choice to the cost model. */
int ggb_batch_set_plan(ggb_batch *b, int window_bits, int team_ctas);
int ggb_batch_get_plan(const ggb_batch *b, int *window_bits, int *team_ctas, int *teams);

/* Times every feasible (window_bits, team_ctas) pair on the batch's current
 * adjacency (iters timed launches each, after one warm-up) and keeps the
 * fastest; reports it and its time. */
int ggb_batch_autotune(ggb_batch *b, int iters, int *window_bits, int *team_ctas, double *best_ms);

/* Device address of graph i's [nodes][degree] adjacency inside the batch
 * (16-byte aligned), for producers that write candidates on the device. */
int ggb_batch_adj_device(ggb_batch *b, int graph, int **adj_dev);

/* Copies host adjacency arrays adj[0..n_graphs) into the batch (on `stream`,
 * or the batch's own stream when NULL). */
int ggb_batch_upload(ggb_batch *b, const int *const *adj, void *stream);

/* Enqueues the evaluation of the batch's device adjacency on `stream` (NULL:
 * the batch's own stream); ggb_batch_collect waits and writes results[i]
 * (results may be NULL to only check for errors). */
int ggb_batch_launch(ggb_batch *b, void *stream);
int ggb_batch_collect(ggb_batch *b, void *stream, ggb_result *results);

/* Upload + launch + collect. */
int ggb_batch_eval(ggb_batch *b, const int *const *adj, ggb_result *results);

/* Device time of the last collected launch (CUDA events around it). */
int ggb_batch_kernel_ms(const ggb_batch *b, double *ms);

/* ---- the proposal filter's network (learned annealing) ------------------ */

/* A 32 -> 256 -> 256 -> 1 ReLU MLP on BF16 tensor cores with FP32
 * accumulation, trained with Adam on the mean squared error.  The annealing
 * engine (ggb_sa_*) owns one; these entry points exist so the network can be
 * checked on its own (host arrays in and out).  Parameters are packed FP32:
 * W1 [256][32], b1 [256], W2 [256][256], b2 [256], w3 [256], b3 [1]
 * (ggb_mlp_param_count() values).  No counterpart in the reference. */
typedef struct ggb_mlp ggb_mlp;
int ggb_mlp_create(int max_rows, unsigned long long seed, ggb_mlp **out);
void ggb_mlp_destroy(ggb_mlp *m);
int ggb_mlp_param_count(void);
int ggb_mlp_set_params(ggb_mlp *m, const float *params);   /* also resets Adam */
int ggb_mlp_get_params(ggb_mlp *m, float *params);
int ggb_mlp_set_adam(ggb_mlp *m, float lr, float beta1, float beta2, float eps);
/* y[r] for rows x 32 FP32 features (rounded to BF16 on the way in);
 * rows % 16 == 0, rows <= max_rows. */
int ggb_mlp_forward_host(ggb_mlp *m, const float *x, int rows, float *y);
/* Uploads x (as ggb_mlp_forward_host does), then times `reps` back-to-back
 * launches of the inference forward on the device-resident rows with CUDA
 * events on one stream; *ms = the mean time of one forward pass. */
int ggb_mlp_time_forward(ggb_mlp *m, const float *x, int rows, int reps, double *ms);
/* Loss and gradients (packed like the parameters) of the mean squared error
 * of rows samples against targets t; rows % 16 == 0, rows <= 256. */
int ggb_mlp_grads_host(ggb_mlp *m, const float *x, const float *t, int rows, float *loss, float *grads);
/* `steps` Adam steps on the same rows; reports the loss of the last one. */
int ggb_mlp_train_host(ggb_mlp *m, const float *x, const float *t, int rows, int steps, float *last_loss);

/* ---- annealing on the device -------------------------------------------- */

/* Simulated annealing of a simple degree-regular general graph (groups = 1,
 * no added centres) with the whole step on the device, replayed as one CUDA
 * graph per step.  Each step draws `proposals` 2-opt swaps of the current
 * graph (general/sa.c:217-369 rules: no self-loop, no repeated edge); when
 * proposals > candidates, the proposal filter's network ranks them and the
 * best `candidates` (a quarter of them drawn at random from the rest) are
 * evaluated exactly in one batch launch, together with four predicted
 * composites: the first m, m/2, m/4, m/8 proposals of the ranking that are
 * predicted to help and have disjoint endpoints, each applied to the current
 * graph as one move.  The strictly improving candidates with disjoint
 * endpoints (at most compose_max) are composed into one more graph, evaluated
 * exactly too; the best of all these exactly evaluated graphs is accepted by
 * the reference's rule (general/sa.c:371-411: smaller diameter,
 * or equal diameter and a distance total not larger, or, when not
 * hill-climbing, exp(diff / temp) > uniform).  With a filter, every step
 * trains the network on the evaluated candidates' exact changes and an
 * accepted move re-profiles the current graph.  candidates = proposals = 1,
 * compose_max = 0 is the reference's plain step.  No host round trip per
 * step; no counterpart for the batching and the filter in the reference. */
typedef struct ggb_sa ggb_sa;

typedef struct ggb_sa_stats {
  long long step, accepts, multi_accepts, moved_swaps, evals;
  long long pred_accepts;            /* accepted predicted composites */
  long long unevaluated;             /* candidates the delta path could not serve (rejected) */
  int cur_diam, best_diam;
  long long cur_total, best_total;   /* exact distance totals (the reference's sum) */
  double cur_aspl, best_aspl;
  double temp;
  int done;                          /* the target was reached */
  int delta;                         /* 1: candidates evaluated against the kept base (exact);
                                        0: in full (plain mode, or graphs where the delta path
                                        would not serve most candidates) */
} ggb_sa_stats;

/* edges: [nodes*degree/2][2] (a simple degree-regular graph, connected).
 * candidates in [1, 256]; proposals = candidates (no filter) or a multiple of
 * 16 up to 4096 (then candidates is a multiple of 16, degree <= 32). */
int ggb_sa_create(int nodes, int degree, const int *edges, int candidates, int proposals, int compose_max,
                  unsigned long long seed, ggb_sa **out);
/* The same for a graph with `groups` rotational symmetry groups (invariant
 * under v -> v + nodes/groups, edges in the reference's symmetric line order:
 * line k*BL + i is line i shifted by k*nodes/groups, general/main.c:175-183).
 * Every move keeps the symmetry: two random lines of different orbits are
 * swapped in every copy (2g-opt, general/sa.c:217-369), two lines of one orbit
 * re-pair that orbit with a random shift (1g-opt, general/common.c:162-276);
 * the four endpoint classes (v mod nodes/groups) must be distinct.  Each
 * candidate is evaluated in full over nodes/groups sources and Metropolis uses
 * the reference's diff = change of the distance total / groups.  No proposal
 * filter (candidates = proposals); groups = 1 is ggb_sa_create. */
int ggb_sa_create_symmetric(int nodes, int degree, int groups, const int *edges, int candidates, int compose_max,
                            unsigned long long seed, ggb_sa **out);
/* Grid graphs without symmetry (grid/sa.c:137-221): vertex v is lattice
 * point (v / height, v % height) and every move keeps both new edges within
 * Manhattan length max_length.  Every current edge must already be within
 * it.  Set before running. */
int ggb_sa_set_grid(ggb_sa *a, int height, int max_length);
void ggb_sa_destroy(ggb_sa *a);
/* Temperature, cooling factor per step, and hill climbing (the reference's
 * -H: accept only when not worse).  Default: hill climbing. */
int ggb_sa_set_schedule(ggb_sa *a, double temp, double cooling_rate, int hill_climbing);
/* With a proposal filter: how many predicted composites each step evaluates
 * (0..8; the default 4) and the largest one's swaps (default 64). */
int ggb_sa_set_predicted(ggb_sa *a, int composites, int max_swaps);
/* Stop (every later step does nothing) once diameter <= diameter and the
 * distance total <= total. */
int ggb_sa_set_target(ggb_sa *a, int diameter, long long total);
/* Autotunes the plan of the candidate batch on the current graph. */
int ggb_sa_autotune(ggb_sa *a, int iters, int *window_bits, int *team_ctas, double *best_ms);
/* Runs `steps` steps and reports the state. */
int ggb_sa_run(ggb_sa *a, long long steps, ggb_sa_stats *stats);
/* Current (best = 0) or best (best = 1) edge list, [lines][2]. */
int ggb_sa_edges(ggb_sa *a, int best, int *edges);
/* With a proposal filter: the network's predictions and the exact labels
 * (scaled change of the distance total) of the last step's `candidates`
 * evaluated swaps; the last quarter of them were drawn at random. */
int ggb_sa_last_step(ggb_sa *a, float *predicted, float *label);
/* Self-check of the delta evaluation (candidates > 1): draws `candidates`
 * fresh swaps of the current graph, evaluates them against the base and in
 * full, and counts the disagreements in diameter, connectivity or distance
 * sum among those the delta path served; dense_windows (may be NULL)
 * receives how many (candidate, window) tasks fell back to a dense sweep. */
int ggb_sa_check_delta(ggb_sa *a, int *compared, int *mismatches, int *unevaluated, int *dense_windows);
/* The kept base's build plan, timed at creation: CTAs per team and teams
 * (0, 0 without a base). */
int ggb_sa_base_plan(const ggb_sa *a, int *team_ctas, int *teams);
/* Per-vertex level statistics of the current graph, [nodes][32]: entry
 * [v][k] = vertices not within distance k of v. */
int ggb_sa_profile(ggb_sa *a, unsigned *stats);

/* Checkpoint and resume of an annealing run.  The reference resumes a run
 * from the graph it wrote with -o, re-read with -M (general/main.c:444-451,
 * 367-373), with a fresh temperature and random stream; a checkpoint here
 * also keeps the step count (which keys the device's counter-based random
 * stream), the temperature and schedule, the counters, the best graph and,
 * with a filter, the network's parameters and Adam state, so that a resumed
 * run continues the interrupted one step for step.  To resume: read the
 * current edges out of the checkpoint (ggb_sa_checkpoint_edges, best = 0),
 * create an annealer from them with the same arguments (and the same
 * ggb_sa_set_predicted / ggb_sa_set_grid calls), then ggb_sa_restore.  Only
 * the library version that wrote a checkpoint reads it. */
long long ggb_sa_checkpoint_bytes(const ggb_sa *a);
int ggb_sa_save(ggb_sa *a, void *buf, long long bytes);
int ggb_sa_restore(ggb_sa *a, const void *buf, long long bytes);
int ggb_sa_checkpoint_info(const void *buf, long long bytes, int *nodes, int *degree, int *groups, int *lines);
/* Current (best = 0) or best (best = 1) edges of a checkpoint, [lines][2]. */
int ggb_sa_checkpoint_edges(const void *buf, long long bytes, int best, int *edges);

#ifdef __cplusplus
}
#endif

/* ---- drop-in shim: general (link libgg_general.so instead of evaluation.o) */
#ifdef GGB_DROPIN_GENERAL
#ifdef __cplusplus
extern "C" {
#endif
/* general/common.h:112-113 and general/evaluation.cu:205-207.  Any algo is
 * evaluated by the bit-parallel path (MATRIX_OP and MATRIX_OP_MEM_SAVING give
 * the same answer; the reference's CUDA evaluation also sends every algo other
 * than MATRIX_OP down its matrix path).  Brackets TIMER_APSP through the
 * host's timer_start/timer_stop when the host defines them. */
bool evaluation(const int nodes, const int based_nodes, const int groups, const int lines,
                const int degree, int *adj, int *diameter, double *ASPL,
                const int added_centers, const int algo);
/* general/main.c:3 and general/evaluation.cu:178: selects GPU rank % gpus
 * and sizes the device buffers. */
void init_matrix_dev(const int nodes, const int degree, const int based_nodes, const int algo);
/* general/main.c:4 and general/evaluation.cu:196. */
void finalize_matrix_dev(void);
#ifdef __cplusplus
}
#endif
#endif

/* ---- drop-in shim: grid (link libgg_grid.so instead of evaluation.o) --- */
#ifdef GGB_DROPIN_GRID
#ifdef __cplusplus
extern "C" {
#endif
/* grid/common.h:88-90.  enable_bfs selects the reference's queue BFS, whose
 * distance total equals the matrix path's; both are served by the GPU path.
 * No init hook exists in the grid program: buffers are created lazily. */
bool evaluation(const int nodes, const int degree, const int groups, const int *adjacency,
                const int based_nodes, const int height, const int based_height, int *diameter,
                double *ASPL, const bool enable_bfs, const int *rotate_hash);
#ifdef __cplusplus
}
#endif
#endif

#endif /* GRAPHGOLF_B200_H */
