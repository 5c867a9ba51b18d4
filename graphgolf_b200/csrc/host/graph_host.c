/*
 * graph_host.c -- host-side graph utilities of graphgolf_b200 (libggb_host.so).
 *
 * Seeded graph generators, the reference's edge-file formats, adjacency
 * construction and graph checks.  All randomness comes from one
 * xoshiro256** stream (Blackman & Vigna, "Scrambled linear pseudorandom
 * number generators", 2018) seeded through splitmix64, so a (generator,
 * parameters, seed) triple names the same graph on every machine.
 *
 * Formats and layouts follow the reference:
 *   general edge file: "a b" per line            (general/main.c:112-126, :311-315)
 *   grid edge file:    "x,y x,y", vertex x*H+y   (grid/main.c:354-376, grid/common.c:53-61)
 *   adjacency rows in edge order                (general/sa.c:61-74, grid/common.c:14-27)
 *   symmetric line order: line j*based_lines+i is line i shifted by j*based_nodes
 *                                               (general/main.c:175-183)
 *   grid rotation relabel                       (grid/common.c:63-86, :312-341)
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define GGB_H_OK 0
#define GGB_H_EINVAL -1
#define GGB_H_ENOMEM -2
#define GGB_H_EFAIL -3
#define GGB_H_EIO -4

/* ---- PRNG ------------------------------------------------------------- */
typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix64(uint64_t *x)
{
  uint64_t z = (*x += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

static void rng_seed(rng_t *r, uint64_t seed)
{
  uint64_t x = seed;
  for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}

static inline uint64_t rotl(const uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t rng_next(rng_t *r)
{
  uint64_t *s = r->s;
  const uint64_t result = rotl(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return result;
}

/* Uniform integer in [0, n) by Lemire's multiply-and-reject. */
static uint32_t rng_below(rng_t *r, uint32_t n)
{
  uint64_t m = (uint64_t)(uint32_t)(rng_next(r) >> 32) * n;
  uint32_t lo = (uint32_t)m;
  if (lo < n) {
    uint32_t thresh = (uint32_t)(-n) % n;
    while (lo < thresh) {
      m = (uint64_t)(uint32_t)(rng_next(r) >> 32) * n;
      lo = (uint32_t)m;
    }
  }
  return (uint32_t)(m >> 32);
}

/* ---- neighbour sets for duplicate checks ------------------------------ */
typedef struct { int n, d; int *nb; int *deg; } nbset_t;

static int nb_init(nbset_t *s, int n, int d)
{
  s->n = n; s->d = d;
  s->nb = malloc(sizeof(int) * (size_t)n * (d > 0 ? d : 1));
  s->deg = calloc((size_t)n, sizeof(int));
  return (s->nb && s->deg) ? 0 : -1;
}
static void nb_free(nbset_t *s) { free(s->nb); free(s->deg); }
static void nb_clear(nbset_t *s) { memset(s->deg, 0, sizeof(int) * (size_t)s->n); }
static int nb_has(const nbset_t *s, int a, int b)
{
  const int *p = s->nb + (size_t)a * s->d;
  for (int i = 0; i < s->deg[a]; i++) if (p[i] == b) return 1;
  return 0;
}
static void nb_add(nbset_t *s, int a, int b)
{
  s->nb[(size_t)a * s->d + s->deg[a]++] = b;
  if (a != b) s->nb[(size_t)b * s->d + s->deg[b]++] = a;
}
static void nb_del1(nbset_t *s, int a, int b)
{
  int *p = s->nb + (size_t)a * s->d;
  for (int i = 0; i < s->deg[a]; i++)
    if (p[i] == b) { p[i] = p[--s->deg[a]]; return; }
}
static void nb_del(nbset_t *s, int a, int b) { nb_del1(s, a, b); if (a != b) nb_del1(s, b, a); }

/* ---- random simple d-regular graph ------------------------------------ */
/*
 * Configuration (pairing) model with per-pair retry: two stubs are drawn from
 * the remaining pool; a self-loop or an edge already present is redrawn.  When
 * the last stubs admit no valid pair, an existing edge (c,e) is rewired with
 * the stuck pair (a,b) into (a,c),(b,e), which keeps every degree.  Whole-graph
 * rejection would almost never succeed at d >= 8.  Edges are written in the
 * order they are created: edges[2*i], edges[2*i+1].
 */
int ggbh_random_regular(int n, int d, uint64_t seed, int *edges)
{
  if (n <= 0 || d < 0 || d >= n || ((long long)n * d) % 2) return GGB_H_EINVAL;
  const long long M = (long long)n * d, lines = M / 2;
  if (M > 0x7fffffffLL) return GGB_H_EINVAL;
  int *pool = malloc(sizeof(int) * (size_t)(M > 0 ? M : 1));
  nbset_t s;
  if (!pool || nb_init(&s, n, d)) { free(pool); nb_free(&s); return GGB_H_ENOMEM; }
  rng_t r;
  rng_seed(&r, seed ^ 0x52414e444f4d52ULL);
  int rc = GGB_H_EFAIL;
  for (int attempt = 0; attempt < 64; attempt++) {
    long long m = M, e = 0;
    for (long long i = 0; i < M; i++) pool[i] = (int)(i / d);
    nb_clear(&s);
    int stuck = 0;
    while (m > 0) {
      int ok = 0;
      for (int tries = 0; tries < 256 && !ok; tries++) {
        uint32_t i = rng_below(&r, (uint32_t)m), j = rng_below(&r, (uint32_t)m);
        if (i == j) continue;
        int a = pool[i], b = pool[j];
        if (a == b || nb_has(&s, a, b)) continue;
        nb_add(&s, a, b);
        edges[2 * e] = a; edges[2 * e + 1] = b; e++;
        /* remove i and j from the pool (larger index first) */
        uint32_t hi = i > j ? i : j, lo = i > j ? j : i;
        pool[hi] = pool[--m];
        pool[lo] = pool[--m];
        ok = 1;
      }
      if (ok) continue;
      /* No valid pair found by sampling: rewire through an existing edge. */
      int a = pool[m - 1], b = pool[m - 2];
      int fixed = 0;
      for (int tries = 0; tries < 4096 && e > 0 && !fixed; tries++) {
        long long k = (long long)rng_below(&r, (uint32_t)e);
        int c = edges[2 * k], f = edges[2 * k + 1];
        if (rng_below(&r, 2)) { int t = c; c = f; f = t; }
        if (a == c || b == f || nb_has(&s, a, c) || nb_has(&s, b, f)) continue;
        nb_del(&s, c, f);
        nb_add(&s, a, c);
        nb_add(&s, b, f);
        edges[2 * k] = a; edges[2 * k + 1] = c;
        edges[2 * e] = b; edges[2 * e + 1] = f; e++;
        m -= 2;
        fixed = 1;
      }
      if (!fixed) { stuck = 1; break; }
    }
    if (!stuck && e == lines) { rc = GGB_H_OK; break; }
  }
  free(pool);
  nb_free(&s);
  return rc;
}

/* ---- rotationally symmetric d-regular graph (general -g) -------------- */
/*
 * A graph on n = g*B vertices invariant under v -> v+B (mod n).  Each base
 * edge (a, b) with a in [0,B) stands for the orbit {(a+jB, b+jB) mod n}, and
 * the edges are written in the reference's line order: line j*based_lines+i
 * is base line i shifted by j*B (general/main.c:175-183), so the reference
 * accepts the file with -M -g g.  Base edges pair vertex classes (v mod B)
 * with per-pair retry, each class appearing d times; the second endpoint gets
 * a random shift k*B.  A base edge whose endpoints differ by n/2 is refused:
 * its orbit would repeat edges.
 */
int ggbh_symmetric_regular(int n, int d, int g, uint64_t seed, int *edges)
{
  if (n <= 0 || d < 0 || g <= 0 || n % g || d >= n) return GGB_H_EINVAL;
  const int B = n / g;
  const long long M = (long long)B * d;
  if (M % 2) return GGB_H_EINVAL;
  const long long based_lines = M / 2;
  int *pool = malloc(sizeof(int) * (size_t)(M > 0 ? M : 1));
  int *base = malloc(sizeof(int) * (size_t)(M > 0 ? M : 1));
  nbset_t s;
  if (!pool || !base || nb_init(&s, n, d)) { free(pool); free(base); nb_free(&s); return GGB_H_ENOMEM; }
  rng_t r;
  rng_seed(&r, seed ^ 0x53594d4d45545259ULL);
  int rc = GGB_H_EFAIL;
  for (int attempt = 0; attempt < 256 && rc; attempt++) {
    long long m = M, e = 0;
    for (long long i = 0; i < M; i++) pool[i] = (int)(i / d);
    nb_clear(&s);
    int stuck = 0;
    while (m > 0 && !stuck) {
      int ok = 0;
      for (int tries = 0; tries < 512 && !ok; tries++) {
        uint32_t i = rng_below(&r, (uint32_t)m), j = rng_below(&r, (uint32_t)m);
        if (i == j) continue;
        int a = pool[i], c = pool[j];
        int k = (int)rng_below(&r, (uint32_t)g);
        int b = c + k * B;
        long long diff = ((long long)b - a) % n;
        if (diff < 0) diff += n;
        if (diff == 0) continue;                      /* self-loop */
        if (n % 2 == 0 && diff == n / 2) continue;    /* short orbit */
        if (nb_has(&s, a, b)) continue;               /* orbit already present */
        for (int jj = 0; jj < g; jj++) {
          int x = (a + jj * B) % n, y = (b + jj * B) % n;
          nb_add(&s, x, y);
        }
        base[2 * e] = a; base[2 * e + 1] = b; e++;
        uint32_t hi = i > j ? i : j, lo = i > j ? j : i;
        pool[hi] = pool[--m];
        pool[lo] = pool[--m];
        ok = 1;
      }
      if (!ok) stuck = 1;
    }
    if (!stuck && e == based_lines) {
      for (int jj = 0; jj < g; jj++)
        for (long long i = 0; i < based_lines; i++) {
          long long line = jj * based_lines + i;
          edges[2 * line] = (int)(((long long)base[2 * i] + (long long)jj * B) % n);
          edges[2 * line + 1] = (int)(((long long)base[2 * i + 1] + (long long)jj * B) % n);
        }
      rc = GGB_H_OK;
    }
  }
  free(pool);
  free(base);
  nb_free(&s);
  return rc;
}

/* ---- length-bounded grid graph ----------------------------------------- */
static int grid_dist(int v, int w, int H)
{
  int dx = v / H - w / H, dy = v % H - w % H;
  return (dx < 0 ? -dx : dx) + (dy < 0 ? -dy : dy);
}

/* Hamiltonian cycle through every lattice point with unit steps (needs W*H
 * even): row 0 left to right, a snake over columns 1..W-1 of rows 1..H-1, and
 * back up column 0.  Written as vertex ids x*H+y. */
static int grid_cycle(int W, int H, int *cyc)
{
  int transpose = 0;
  if (H % 2) {
    if (W % 2) return -1;
    transpose = 1;
    int t = W; W = H; H = t;
  }
  int k = 0;
#define PUT(x, y) cyc[k++] = transpose ? ((y) * W + (x)) : ((x) * H + (y))
  for (int x = 0; x < W; x++) PUT(x, 0);
  for (int y = 1; y < H; y++) {
    if (y % 2) for (int x = W - 1; x >= 1; x--) PUT(x, y);
    else for (int x = 1; x < W; x++) PUT(x, y);
  }
  for (int y = H - 1; y >= 1; y--) PUT(0, y);
#undef PUT
  return k;
}

static int connected(int n, int lines, const int *edges)
{
  int *deg = calloc((size_t)n + 1, sizeof(int)), *adj = malloc(sizeof(int) * (size_t)(2 * lines + 1));
  int *q = malloc(sizeof(int) * (size_t)n);
  char *seen = calloc((size_t)n, 1);
  if (!deg || !adj || !q || !seen) { free(deg); free(adj); free(q); free(seen); return -1; }
  for (int i = 0; i < lines; i++) { deg[edges[2 * i] + 1]++; deg[edges[2 * i + 1] + 1]++; }
  for (int v = 0; v < n; v++) deg[v + 1] += deg[v];
  int *fill = calloc((size_t)n, sizeof(int));
  if (!fill) { free(deg); free(adj); free(q); free(seen); return -1; }
  for (int i = 0; i < lines; i++) {
    int a = edges[2 * i], b = edges[2 * i + 1];
    adj[deg[a] + fill[a]++] = b;
    adj[deg[b] + fill[b]++] = a;
  }
  int head = 0, tail = 0;
  seen[0] = 1; q[tail++] = 0;
  while (head < tail) {
    int v = q[head++];
    for (int i = deg[v]; i < deg[v + 1]; i++)
      if (!seen[adj[i]]) { seen[adj[i]] = 1; q[tail++] = adj[i]; }
  }
  free(deg); free(adj); free(q); free(seen); free(fill);
  return tail == n;
}

/*
 * A d-regular graph on the W x H lattice whose every edge has Manhattan length
 * <= R: the (d/2)-th power of a unit-step Hamiltonian cycle (edges of length
 * <= d/2 <= R), then `swaps` local 2-opt exchanges, then more until the graph
 * is connected.  An exchange takes an edge (a,b), a vertex c within distance
 * R of a and an edge (c,f), and rewires them to (a,c),(b,f) when (b,f) is no
 * longer than R and neither new edge exists; degrees never change.  Drawing c
 * near a keeps the acceptance rate high, so the lattice structure is mixed
 * well beyond the starting cycle.  d must be even, W*H even, d/2 <= R and
 * W*H > d.  Edges are written sorted by their smaller endpoint.
 */
int ggbh_grid_regular(int W, int H, int d, int R, long long swaps, uint64_t seed, int *edges)
{
  if (W <= 0 || H <= 0 || d <= 0 || d % 2 || R <= 0 || d / 2 > R) return GGB_H_EINVAL;
  const int n = W * H;
  if (n % 2 || n <= d) return GGB_H_EINVAL;
  const int lines = n * d / 2;
  int *cyc = malloc(sizeof(int) * (size_t)n);
  nbset_t s;
  if (!cyc || nb_init(&s, n, d)) { free(cyc); nb_free(&s); return GGB_H_ENOMEM; }
  if (grid_cycle(W, H, cyc) != n) { free(cyc); nb_free(&s); return GGB_H_EINVAL; }
  for (int step = 1; step <= d / 2; step++)
    for (int i = 0; i < n; i++) {
      int a = cyc[i], b = cyc[(i + step) % n];
      if (nb_has(&s, a, b)) { free(cyc); nb_free(&s); return GGB_H_EFAIL; }
      nb_add(&s, a, b);
    }
  free(cyc);
  rng_t r;
  rng_seed(&r, seed ^ 0x4752494447524944ULL);
  long long todo = swaps;
  int rc = GGB_H_EFAIL;
  for (int round = 0; round < 1000 && rc; round++) {
    for (long long it = 0; it < todo; it++) {
      int a = (int)rng_below(&r, (uint32_t)n);
      int b = s.nb[(size_t)a * d + rng_below(&r, (uint32_t)d)];
      int ax = a / H, ay = a % H;
      int cx = ax + (int)rng_below(&r, (uint32_t)(2 * R + 1)) - R;
      int cy = ay + (int)rng_below(&r, (uint32_t)(2 * R + 1)) - R;
      if (cx < 0 || cy < 0 || cx >= W || cy >= H) continue;
      int c = cx * H + cy;
      if (grid_dist(a, c, H) > R) continue;
      int f = s.nb[(size_t)c * d + rng_below(&r, (uint32_t)d)];
      if (c == a || c == b || f == a || f == b) continue;
      if (grid_dist(b, f, H) > R) continue;
      if (nb_has(&s, a, c) || nb_has(&s, b, f)) continue;
      nb_del(&s, a, b); nb_del(&s, c, f);
      nb_add(&s, a, c); nb_add(&s, b, f);
    }
    int e = 0;
    for (int v = 0; v < n; v++)
      for (int k = 0; k < d; k++) {
        int u = s.nb[(size_t)v * d + k];
        if (u > v) { edges[2 * e] = v; edges[2 * e + 1] = u; e++; }
      }
    int c = connected(n, lines, edges);
    if (c < 0) { rc = GGB_H_ENOMEM; break; }
    if (c) rc = GGB_H_OK;
    todo = lines;
  }
  nb_free(&s);
  return rc;
}

/* ---- adjacency ---------------------------------------------------------- */
/* general/sa.c:61-74 and grid/common.c:14-27: row v lists v's neighbours in
 * edge order.  Returns GGB_H_EINVAL if some vertex does not have exactly d. */
int ggbh_create_adj(int n, int lines, int d, const int *edges, int *adj)
{
  int *count = calloc((size_t)n, sizeof(int));
  if (!count) return GGB_H_ENOMEM;
  int rc = GGB_H_OK;
  for (int i = 0; i < lines && !rc; i++) {
    int a = edges[2 * i], b = edges[2 * i + 1];
    if (a < 0 || a >= n || b < 0 || b >= n || count[a] >= d || count[b] >= d) { rc = GGB_H_EINVAL; break; }
    adj[(size_t)a * d + count[a]++] = b;
    adj[(size_t)b * d + count[b]++] = a;
  }
  for (int v = 0; v < n && !rc; v++) if (count[v] != d) rc = GGB_H_EINVAL;
  free(count);
  return rc;
}

/* ---- grid rotation relabel --------------------------------------------- */
/* ROTATE of grid/common.c:63-86 (v = x*height + y). */
static int rotate(int v, int height, int width, int groups, int degree)
{
  int w = v / height, h = v % height;
  if (groups == 2) return (width - w - 1) * height + (height - h - 1);
  if (degree == 90) return h * height + (height - w - 1);
  if (degree == 180) return (height - w - 1) * height + (height - h - 1);
  return (height - h - 1) * height + w;
}

/* create_rotate_hash of grid/common.c:312-341. */
int ggbh_rotate_hash(int n, int height, int width, int groups, int *rh)
{
  if (n <= 0 || (groups != 1 && groups != 2 && groups != 4) || n % groups) return GGB_H_EINVAL;
  const int based = n / groups;
  if (groups == 1) {
    for (int i = 0; i < based; i++) rh[i] = i;
    return GGB_H_OK;
  }
  const int bh = height / 2;
  for (int i = 0; i < based; i++) {
    int j = (i / bh) * height + (i % bh);
    rh[j] = i;
    if (groups == 2) {
      rh[rotate(j, height, width, 2, 180)] = i + based;
    } else {
      rh[rotate(j, height, width, 4, 90)] = i + based;
      rh[rotate(j, height, width, 4, 180)] = i + based * 2;
      rh[rotate(j, height, width, 4, 270)] = i + based * 3;
    }
  }
  return GGB_H_OK;
}

/* ---- edge files --------------------------------------------------------- */
/* Number of lines (newline characters), as count_lines (general/main.c:97-110). */
long long ggbh_count_lines(const char *path)
{
  FILE *fp = fopen(path, "r");
  if (!fp) return GGB_H_EIO;
  long long lines = 0;
  int c;
  while ((c = fgetc(fp)) != EOF) if (c == '\n') lines++;
  fclose(fp);
  return lines;
}

/* "a b" lines, as read_file (general/main.c:112-126).  Returns edges read. */
long long ggbh_read_general(const char *path, int *edges, long long max_lines)
{
  FILE *fp = fopen(path, "r");
  if (!fp) return GGB_H_EIO;
  long long i = 0;
  int a, b;
  while (i < max_lines && fscanf(fp, "%d %d", &a, &b) == 2) { edges[2 * i] = a; edges[2 * i + 1] = b; i++; }
  fclose(fp);
  return i;
}

int ggbh_write_general(const char *path, long long lines, const int *edges)
{
  FILE *fp = fopen(path, "w");
  if (!fp) return GGB_H_EIO;
  for (long long i = 0; i < lines; i++) fprintf(fp, "%d %d\n", edges[2 * i], edges[2 * i + 1]);
  return fclose(fp) ? GGB_H_EIO : GGB_H_OK;
}

/* "x,y x,y" lines, as read_file_lattice (grid/main.c:354-376): the height is
 * one more than the largest y, vertex ids are x*height+y.  Returns edges read
 * and the width/height through the pointers. */
long long ggbh_read_grid(const char *path, int *edges, long long max_lines, int *width, int *height)
{
  FILE *fp = fopen(path, "r");
  if (!fp) return GGB_H_EIO;
  int p[4], w = 0, h = 0;
  while (fscanf(fp, "%d,%d %d,%d", &p[0], &p[1], &p[2], &p[3]) == 4) {
    if (p[0] > w) w = p[0];
    if (p[2] > w) w = p[2];
    if (p[1] > h) h = p[1];
    if (p[3] > h) h = p[3];
  }
  w += 1; h += 1;
  rewind(fp);
  long long i = 0;
  while (i < max_lines && fscanf(fp, "%d,%d %d,%d", &p[0], &p[1], &p[2], &p[3]) == 4) {
    edges[2 * i] = p[0] * h + p[1];
    edges[2 * i + 1] = p[2] * h + p[3];
    i++;
  }
  fclose(fp);
  *width = w;
  *height = h;
  return i;
}

int ggbh_write_grid(const char *path, long long lines, const int *edges, int height)
{
  FILE *fp = fopen(path, "w");
  if (!fp) return GGB_H_EIO;
  for (long long i = 0; i < lines; i++)
    fprintf(fp, "%d,%d %d,%d\n", edges[2 * i] / height, edges[2 * i] % height, edges[2 * i + 1] / height,
            edges[2 * i + 1] % height);
  return fclose(fp) ? GGB_H_EIO : GGB_H_OK;
}

/* ---- checks ------------------------------------------------------------- */
/* verfy_graph essentials (general/main.c:212-241, grid/main.c:428-451): every
 * vertex has degree d, no self-loop, no repeated edge, and (max_len > 0) every
 * grid edge no longer than max_len.  Returns 0 if valid, else a code 1..4. */
int ggbh_verify(int n, long long lines, int d, const int *edges, int max_len, int height)
{
  nbset_t s;
  if (nb_init(&s, n, d)) { nb_free(&s); return GGB_H_ENOMEM; }
  int rc = 0;
  for (long long i = 0; i < lines && !rc; i++) {
    int a = edges[2 * i], b = edges[2 * i + 1];
    if (a < 0 || b < 0 || a >= n || b >= n) rc = 1;
    else if (a == b) rc = 2;
    else if (s.deg[a] >= d || s.deg[b] >= d) rc = 1;
    else if (nb_has(&s, a, b)) rc = 3;
    else if (max_len > 0 && grid_dist(a, b, height) > max_len) rc = 4;
    else nb_add(&s, a, b);
  }
  for (int v = 0; v < n && !rc; v++) if (s.deg[v] != d) rc = 1;
  nb_free(&s);
  return rc;
}
