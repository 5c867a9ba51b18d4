"""Seeded graphs, edge files and adjacency (wrappers of libggb_host.so).

Every generator is deterministic in (parameters, seed) on every machine: the
randomness is the library's own xoshiro256** stream, not libc's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import load

_ERR = {-1: "invalid arguments", -2: "out of memory", -3: "generator gave up", -4: "I/O error"}


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _check(rc: int, what: str) -> None:
    if rc < 0:
        raise ValueError(f"{what}: {_ERR.get(rc, rc)}")


@dataclass
class Graph:
    """An edge list in the reference's line order plus its adjacency."""

    nodes: int
    degree: int
    edges: np.ndarray          # int32 [lines, 2]
    adj: np.ndarray            # int32 [nodes, degree], rows in edge order
    groups: int = 1            # rotational symmetry groups (general -g / grid -g)
    width: int = 0             # grid only
    height: int = 0            # grid only
    rotate_hash: np.ndarray | None = None   # grid only

    @property
    def lines(self) -> int:
        return int(self.edges.shape[0])

    @property
    def based_nodes(self) -> int:
        return self.nodes // self.groups


def create_adj(nodes: int, degree: int, edges: np.ndarray) -> np.ndarray:
    """general/sa.c:61-74: row v lists v's neighbours in edge order."""
    e = np.ascontiguousarray(edges, dtype=np.int32)
    adj = np.empty((nodes, max(degree, 0)), dtype=np.int32)
    _check(load("host").ggbh_create_adj(nodes, e.shape[0], degree, _ptr(e), _ptr(adj)), "create_adj")
    return adj


def random_regular(nodes: int, degree: int, seed: int) -> Graph:
    """Random simple degree-regular graph (pairing model, per-pair retry)."""
    e = np.empty((nodes * degree // 2, 2), dtype=np.int32)
    _check(load("host").ggbh_random_regular(nodes, degree, seed, _ptr(e)), "random_regular")
    return Graph(nodes, degree, e, create_adj(nodes, degree, e))


def symmetric_regular(nodes: int, degree: int, groups: int, seed: int) -> Graph:
    """Graph invariant under v -> v + nodes/groups, lines in the reference's
    symmetric order (accepted by the reference with -M -g groups)."""
    e = np.empty((nodes * degree // 2, 2), dtype=np.int32)
    _check(load("host").ggbh_symmetric_regular(nodes, degree, groups, seed, _ptr(e)), "symmetric_regular")
    return Graph(nodes, degree, e, create_adj(nodes, degree, e), groups=groups)


def rotate_hash(nodes: int, height: int, width: int, groups: int) -> np.ndarray:
    """create_rotate_hash (grid/common.c:312-341)."""
    rh = np.empty(nodes, dtype=np.int32)
    _check(load("host").ggbh_rotate_hash(nodes, height, width, groups, _ptr(rh)), "rotate_hash")
    return rh


def grid_regular(width: int, height: int, degree: int, length: int, seed: int,
                 swaps: int | None = None) -> Graph:
    """Degree-regular graph on the width x height lattice, every edge of
    Manhattan length <= length; vertex ids x*height + y (grid/common.c:53-61)."""
    n = width * height
    lines = n * degree // 2
    e = np.empty((lines, 2), dtype=np.int32)
    sw = 20 * lines if swaps is None else swaps
    _check(load("host").ggbh_grid_regular(width, height, degree, length, sw, seed, _ptr(e)), "grid_regular")
    return Graph(n, degree, e, create_adj(n, degree, e), width=width, height=height,
                 rotate_hash=rotate_hash(n, height, width, 1))


def read_general(path: str, groups: int = 1) -> Graph:
    """Reads a general edge file as the reference does with -M (general/main.c:361-376)."""
    h = load("host")
    lines = h.ggbh_count_lines(path.encode())
    _check(int(lines), f"read {path}")
    e = np.empty((max(lines, 1), 2), dtype=np.int32)
    got = h.ggbh_read_general(path.encode(), _ptr(e), lines)
    _check(int(got), f"read {path}")
    e = e[:got]
    nodes = int(e.max()) + 1
    degree = 2 * got // nodes
    return Graph(nodes, degree, e, create_adj(nodes, degree, e), groups=groups)


def write_general(path: str, g: Graph) -> None:
    e = np.ascontiguousarray(g.edges, dtype=np.int32)
    _check(load("host").ggbh_write_general(path.encode(), e.shape[0], _ptr(e)), f"write {path}")


def read_grid(path: str) -> Graph:
    """Reads "x,y x,y" lines (grid/main.c:354-376); g = 1."""
    h = load("host")
    lines = h.ggbh_count_lines(path.encode())
    _check(int(lines), f"read {path}")
    e = np.empty((max(lines, 1), 2), dtype=np.int32)
    w, hh = C.c_int(0), C.c_int(0)
    got = h.ggbh_read_grid(path.encode(), _ptr(e), lines, C.byref(w), C.byref(hh))
    _check(int(got), f"read {path}")
    e = e[:got]
    n = w.value * hh.value
    degree = 2 * got // n
    return Graph(n, degree, e, create_adj(n, degree, e), width=w.value, height=hh.value,
                 rotate_hash=rotate_hash(n, hh.value, w.value, 1))


def write_grid(path: str, g: Graph) -> None:
    e = np.ascontiguousarray(g.edges, dtype=np.int32)
    _check(load("host").ggbh_write_grid(path.encode(), e.shape[0], _ptr(e), g.height), f"write {path}")


def verify(g: Graph, max_len: int = 0) -> int:
    """0 if regular, loop-free, duplicate-free (and length-bounded); else 1..4."""
    e = np.ascontiguousarray(g.edges, dtype=np.int32)
    return int(load("host").ggbh_verify(g.nodes, e.shape[0], g.degree, _ptr(e), max_len, g.height))


def nonregular(g: Graph, drop: int, seed: int, pad: int = -1) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Removes `drop` seeded random edges from g and returns (edges, adj,
    degrees): adj is [nodes][g.degree] with each row's neighbours first in
    edge order (as the non-regular programs' create_adj) and `pad` in the
    unused slots (pad < 0 means the row's own id, a valid vertex)."""
    rng = np.random.default_rng(seed)
    keep = np.ones(g.lines, dtype=bool)
    keep[rng.choice(g.lines, size=drop, replace=False)] = False
    edges = np.ascontiguousarray(g.edges[keep], dtype=np.int32)
    n, d = g.nodes, g.degree
    adj = np.empty((n, d), dtype=np.int32)
    adj[:] = np.arange(n, dtype=np.int32)[:, None] if pad < 0 else pad
    deg = np.zeros(n, dtype=np.int32)
    for a, b in edges:
        adj[a, deg[a]] = b
        deg[a] += 1
        adj[b, deg[b]] = a
        deg[b] += 1
    return edges, adj, deg



def swap_2opt(g: Graph, seed: int, tries: int = 10000) -> Graph:
    """One seeded 2-opt edge swap of g (the move of general/sa.c:217-369 with
    groups = 1): lines i != j, (a,b),(c,d) become (a,c),(b,d) or (a,d),(b,c),
    redrawn until the result has no self-loop and no repeated edge."""
    rng = np.random.default_rng(seed)
    e = np.array(g.edges, dtype=np.int32, copy=True)
    for _ in range(tries):
        i, j = (int(x) for x in rng.integers(0, g.lines, 2))
        if i == j:
            continue
        a, b = (int(x) for x in e[i])
        c, d = (int(x) for x in e[j])
        (p, q), (r, s) = ((a, c), (b, d)) if rng.integers(2) else ((a, d), (b, c))
        if p == q or r == s or {p, q} == {r, s}:
            continue
        if q in g.adj[p] or s in g.adj[r]:
            continue
        e[i] = (p, q)
        e[j] = (r, s)
        return Graph(g.nodes, g.degree, e, create_adj(g.nodes, g.degree, e), groups=g.groups)
    raise ValueError("swap_2opt: no valid swap found")


def batch_workload(candidates: int = 256, degree: int = 12, n_lo: int = 512, n_hi: int = 16384,
                   base_nodes: int = 4096, seed: int = 1) -> list[Graph]:
    """A mixed batch: a random degree-regular base graph of base_nodes
    vertices, then `candidates` graphs, each one seeded 2-opt swap of its own
    random degree-regular base graph whose vertex count is drawn
    log-uniformly from [n_lo, n_hi]."""
    rng = np.random.default_rng(seed)
    out = [random_regular(base_nodes, degree, seed)]
    for k in range(candidates):
        n = int(round(float(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))))
        if (n * degree) % 2:
            n += 1
        s = seed * 1000003 + k + 1
        out.append(swap_2opt(random_regular(n, degree, s), s))
    return out
