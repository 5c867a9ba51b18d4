// stage_plan.h -- how stage.cu cuts an upload into claimable units.
//
// Host-only and free of CUDA types, so the planning can be checked on its own
// (tests/stage_plan/check.cc).  An upload is a list of segments: source
// arrays that fill ints [off, off + n) of one pinned buffer, in increasing,
// non-overlapping order, with possible gaps between them.  A unit is a
// contiguous range [lo, hi) of that buffer plus the pieces of segments that
// lie in it; the units tile [0, total) without gaps, every unit but the last
// spans at least `chunk` ints, and no piece is longer than `chunk`.
#pragma once
#include <algorithm>
#include <cstddef>
#include <vector>

namespace ggb {

struct StagePiece {
  const int* src;
  size_t off;
  size_t n;
};

struct StageUnit {
  size_t lo, hi;   // ints [lo, hi) of the buffer, sent in one DMA
  int p0, p1;      // pieces [p0, p1) copied before it
};

template <class Seg>
void stage_plan(const Seg* segs, int nsegs, size_t total, size_t chunk, std::vector<StagePiece>& pieces,
                std::vector<StageUnit>& units) {
  pieces.clear();
  units.clear();
  size_t lo = 0;   // first int of the open unit
  int p0 = 0;      // its first piece
  auto close = [&](size_t hi) {
    units.push_back({lo, hi, p0, (int)pieces.size()});
    lo = hi;
    p0 = (int)pieces.size();
  };
  for (int s = 0; s < nsegs; ++s) {
    for (size_t o = 0; o < segs[s].n;) {
      const size_t pos = segs[s].off + o;
      if (pos - lo >= chunk) close(pos);   // a gap before this segment filled the unit
      const size_t m = std::min(segs[s].n - o, chunk - (pos - lo));
      pieces.push_back({segs[s].src + o, pos, m});
      o += m;
      if (pos + m - lo >= chunk) close(pos + m);
    }
  }
  if (lo < total) close(total);
}

}  // namespace ggb
