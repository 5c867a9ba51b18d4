// Checks ggb::stage_plan() (graphgolf_b200/csrc/stage_plan.h) on seeded
// random uploads: segments of random sizes with random gaps, chunks from 1
// int to larger than the whole upload.  For every plan: the units tile
// [0, total) in order, every unit but the last spans at least `chunk` ints,
// every piece lies inside its unit and is at most `chunk` long, and the
// pieces cover each segment exactly once, in order, from the right source.
// Prints "ok <plans>" and exits 0, or the first violation and exits 1.
#include <cstdio>
#include <cstdint>
#include <vector>

#include "stage_plan.h"

struct Seg {
  const int* src;
  size_t off;
  size_t n;
};

static uint64_t rng = 0x9E3779B97F4A7C15ull;
static uint64_t next_u64() {
  rng ^= rng << 13;
  rng ^= rng >> 7;
  rng ^= rng << 17;
  return rng;
}
static size_t below(size_t n) { return n ? (size_t)(next_u64() % n) : 0; }

#define CHECK(c, ...)                        \
  do {                                       \
    if (!(c)) {                              \
      std::printf("plan %d: ", plan);        \
      std::printf(__VA_ARGS__);              \
      std::printf("\n");                     \
      return 1;                              \
    }                                        \
  } while (0)

int main() {
  static int pool[1 << 20];
  int plans = 0;
  for (int plan = 0; plan < 4000; ++plan, ++plans) {
    const int nsegs = (int)below(40);
    std::vector<Seg> segs;
    size_t pos = 0;
    for (int s = 0; s < nsegs; ++s) {
      pos += below(4) == 0 ? below(300) : 0;              // a gap, sometimes
      const size_t n = below(5) == 0 ? 0 : 1 + below(below(2) ? 50 : 1500);
      segs.push_back({pool + below(1000), pos, n});
      pos += n;
    }
    const size_t total = pos + below(3) * below(200);     // a tail after the last segment, sometimes
    const size_t chunks[] = {1, 3, 7, 64, 1000, 4096, 100000};
    const size_t chunk = chunks[below(7)];
    std::vector<ggb::StagePiece> pieces;
    std::vector<ggb::StageUnit> units;
    ggb::stage_plan(segs.data(), nsegs, total, chunk, pieces, units);
    size_t lo = 0;
    int p = 0;
    for (size_t u = 0; u < units.size(); ++u) {
      const ggb::StageUnit& un = units[u];
      CHECK(un.lo == lo, "unit %zu starts at %zu, want %zu", u, un.lo, lo);
      CHECK(un.hi > un.lo, "unit %zu is empty", u);
      CHECK(u + 1 == units.size() || un.hi - un.lo >= chunk, "unit %zu spans %zu < chunk %zu", u,
            un.hi - un.lo, chunk);
      CHECK(un.p0 == p && un.p1 >= un.p0, "unit %zu pieces [%d, %d), want from %d", u, un.p0, un.p1, p);
      for (int k = un.p0; k < un.p1; ++k) {
        const ggb::StagePiece& pc = pieces[k];
        CHECK(pc.n >= 1 && pc.n <= chunk, "piece %d has %zu ints (chunk %zu)", k, pc.n, chunk);
        CHECK(pc.off >= un.lo && pc.off + pc.n <= un.hi, "piece %d [%zu, %zu) outside unit [%zu, %zu)", k,
              pc.off, pc.off + pc.n, un.lo, un.hi);
      }
      lo = un.hi;
      p = un.p1;
    }
    CHECK(lo == total, "units end at %zu, total %zu", lo, total);
    CHECK(p == (int)pieces.size(), "%zu pieces, units cover %d", pieces.size(), p);
    int k = 0;
    for (const Seg& s : segs) {
      size_t o = 0;
      while (o < s.n) {
        CHECK(k < (int)pieces.size(), "segment at %zu not covered", s.off);
        const ggb::StagePiece& pc = pieces[k++];
        CHECK(pc.off == s.off + o && pc.src == s.src + o, "piece %d at %zu, want %zu", k - 1, pc.off, s.off + o);
        o += pc.n;
      }
      CHECK(o == s.n, "segment at %zu overrun", s.off);
    }
    CHECK(k == (int)pieces.size(), "stray pieces");
  }
  std::printf("ok %d\n", plans);
  return 0;
}
