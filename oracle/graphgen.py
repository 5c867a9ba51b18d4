"""Pure-Python copy of the package's seeded graph generators (TEST
INFRASTRUCTURE ONLY).

bench.py's reference arm times the reference's own evaluator on the bench
graph and must not load any of this repository's native libraries, so it
cannot ask libggb_host.so (graphgolf_b200/csrc/host/graph_host.c) for the
graph.  This module draws the same graphs in plain Python: the same
xoshiro256** stream seeded through splitmix64 (Blackman & Vigna, "Scrambled
linear pseudorandom number generators", 2018), the same Lemire
multiply-and-reject bounded draws and the same per-pair-retry pairing model,
in the same order, so a (generator, parameters, seed) triple gives the
identical edge list.  tests/test_graphs.py checks that against the C
generator and against the adjacency hashes of the golden cases.
"""
from __future__ import annotations

import numpy as np

_M64 = (1 << 64) - 1


class _Xoshiro:
    __slots__ = ("s0", "s1", "s2", "s3")

    def __init__(self, seed: int):
        x = seed & _M64
        s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & _M64
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
            s.append(z ^ (z >> 31))
        self.s0, self.s1, self.s2, self.s3 = s

    def next(self) -> int:
        s0, s1, s2, s3 = self.s0, self.s1, self.s2, self.s3
        r = ((s1 * 5) & _M64)
        r = (((r << 7) | (r >> 57)) & _M64) * 9 & _M64
        t = (s1 << 17) & _M64
        s2 ^= s0
        s3 ^= s1
        s1 ^= s2
        s0 ^= s3
        s2 ^= t
        s3 = ((s3 << 45) | (s3 >> 19)) & _M64
        self.s0, self.s1, self.s2, self.s3 = s0, s1, s2, s3
        return r

    def below(self, n: int) -> int:
        """Uniform integer in [0, n) (Lemire's multiply-and-reject on the top 32 bits)."""
        m = (self.next() >> 32) * n
        lo = m & 0xFFFFFFFF
        if lo < n:
            thresh = ((1 << 32) - n) % n
            while lo < thresh:
                m = (self.next() >> 32) * n
                lo = m & 0xFFFFFFFF
        return m >> 32


def random_regular_edges(n: int, d: int, seed: int) -> np.ndarray:
    """Edge list [n*d/2][2] of the seeded random simple d-regular graph that
    graphgolf_b200.graphs.random_regular(n, d, seed) returns."""
    if n <= 0 or d < 0 or d >= n or (n * d) % 2:
        raise ValueError("need 0 <= d < n and n*d even")
    M = n * d
    lines = M // 2
    r = _Xoshiro(seed ^ 0x52414E444F4D52)
    for _attempt in range(64):
        pool = [i // d for i in range(M)]
        nb = [[] for _ in range(n)]
        edges = []
        m = M
        stuck = False
        while m > 0:
            ok = False
            for _tries in range(256):
                i, j = r.below(m), r.below(m)
                if i == j:
                    continue
                a, b = pool[i], pool[j]
                if a == b or b in nb[a]:
                    continue
                nb[a].append(b)
                nb[b].append(a)
                edges.append([a, b])
                hi, lo = (i, j) if i > j else (j, i)
                m -= 1
                pool[hi] = pool[m]
                m -= 1
                pool[lo] = pool[m]
                ok = True
                break
            if ok:
                continue
            a, b = pool[m - 1], pool[m - 2]
            fixed = False
            for _tries in range(4096):
                if not edges:
                    break
                k = r.below(len(edges))
                c, f = edges[k]
                if r.below(2):
                    c, f = f, c
                if a == c or b == f or c in nb[a] or f in nb[b]:
                    continue
                nb[c].remove(f)
                nb[f].remove(c)
                nb[a].append(c)
                nb[c].append(a)
                nb[b].append(f)
                nb[f].append(b)
                edges[k] = [a, c]
                edges.append([b, f])
                m -= 2
                fixed = True
                break
            if not fixed:
                stuck = True
                break
        if not stuck and len(edges) == lines:
            return np.asarray(edges, dtype=np.int32).reshape(lines, 2)
    raise RuntimeError("random_regular: no graph after 64 attempts")


def symmetric_regular_edges(n: int, d: int, g: int, seed: int) -> np.ndarray:
    """Edge list of graphgolf_b200.graphs.symmetric_regular(n, d, g, seed):
    invariant under v -> v + n/g, lines in the reference's symmetric order."""
    if n <= 0 or d < 0 or g <= 0 or n % g or d >= n:
        raise ValueError("bad sizes")
    B = n // g
    M = B * d
    if M % 2:
        raise ValueError("n/g * d must be even")
    based_lines = M // 2
    r = _Xoshiro(seed ^ 0x53594D4D45545259)
    for _attempt in range(256):
        pool = [i // d for i in range(M)]
        nb = [set() for _ in range(n)]
        base = []
        m = M
        stuck = False
        while m > 0 and not stuck:
            ok = False
            for _tries in range(512):
                i, j = r.below(m), r.below(m)
                if i == j:
                    continue
                a, c = pool[i], pool[j]
                k = r.below(g)
                b = c + k * B
                diff = (b - a) % n
                if diff == 0:
                    continue
                if n % 2 == 0 and diff == n // 2:
                    continue
                if b in nb[a]:
                    continue
                for jj in range(g):
                    x, y = (a + jj * B) % n, (b + jj * B) % n
                    nb[x].add(y)
                    nb[y].add(x)
                base.append((a, b))
                hi, lo = (i, j) if i > j else (j, i)
                m -= 1
                pool[hi] = pool[m]
                m -= 1
                pool[lo] = pool[m]
                ok = True
                break
            if not ok:
                stuck = True
        if not stuck and len(base) == based_lines:
            bs = np.asarray(base, dtype=np.int64).reshape(based_lines, 2)
            out = np.concatenate([(bs + jj * B) % n for jj in range(g)]).astype(np.int32)
            return out
    raise RuntimeError("symmetric_regular: no graph after 256 attempts")


def create_adj(n: int, d: int, edges: np.ndarray) -> np.ndarray:
    """general/sa.c:61-74: row v lists v's neighbours in edge order."""
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    src = e.ravel()                 # a0 b0 a1 b1 ...: each line fills a's row, then b's
    dst = e[:, ::-1].ravel()
    cnt = np.bincount(src, minlength=n)
    if cnt.shape[0] != n or not np.all(cnt == d):
        raise ValueError("edge list is not d-regular")
    order = np.argsort(src, kind="stable")
    return dst[order].astype(np.int32).reshape(n, d)
