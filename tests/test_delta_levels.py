"""The two rules by which the delta evaluation decides levels without a sweep
(graphgolf_b200/csrc/apsp_delta.cuh, delta_kernel), checked on the CPU with
plain bitset breadth-first searches over random regular graphs and seeded
2-opt swaps:

- shared levels: S'_k = S_k for every k <= m, where m is the distance from
  the window's sources (swap endpoints masked out) to the nearest endpoint,
  read as the first level at which some endpoint's base row meets the
  window;
- settled tail: once no row differs (D_k empty) and every endpoint's row is
  full, every later level equals the base's.

The GPU tests prove the kernel equal to the full evaluation; these pin the
two rules themselves on small cases, with no GPU."""
import numpy as np
import pytest

from graphgolf_b200 import graphs


def _levels(adj, src):
    """S_k (bool [N][len(src)]) for k = 0, 1, ... until every row is full."""
    n = adj.shape[0]
    s = np.zeros((n, len(src)), dtype=bool)
    s[src, np.arange(len(src))] = True
    out = [s]
    while not s.all() and len(out) <= n:
        t = s.copy()
        for j in range(adj.shape[1]):
            t |= s[adj[:, j]]
        s = t
        out.append(s)
    return out


def _pad(levels, k):
    return levels[min(k, len(levels) - 1)]


@pytest.mark.parametrize("n,d,seed", [(300, 3, 1), (500, 5, 2), (800, 8, 3)])
def test_level_skipping_rules(n, d, seed):
    g = graphs.random_regular(n, d, seed)
    checked_shared = checked_tail = 0
    for t in range(6):
        h = graphs.swap_2opt(g, 1000 * seed + t)
        ends = np.nonzero((h.adj != g.adj).any(axis=1))[0]
        assert len(ends) == 4
        for w0 in range(0, n, 128):
            src = np.array([s for s in range(w0, min(n, w0 + 128)) if s not in set(ends.tolist())])
            if len(src) == 0:
                continue
            base, cand = _levels(g.adj, src), _levels(h.adj, src)
            top = max(len(base), len(cand))
            # shared levels: m = first level at which an endpoint's base row meets the window
            m = next(k for k in range(1, top + 1) if _pad(base, k)[ends].any())
            for k in range(m + 1):
                assert np.array_equal(_pad(base, k), _pad(cand, k)), (t, w0, k, m)
                checked_shared += 1
            # settled tail: D_k empty and every endpoint's row full => equal from then on
            for k in range(top):
                b, c = _pad(base, k), _pad(cand, k)
                if np.array_equal(b, c) and b[ends].all():
                    for k2 in range(k, top + 1):
                        assert np.array_equal(_pad(base, k2), _pad(cand, k2)), (t, w0, k, k2)
                    checked_tail += 1
                    break
    assert checked_shared > 0 and checked_tail > 0
