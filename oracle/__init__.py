"""Test oracle for graphgolf_b200 (TEST INFRASTRUCTURE ONLY).

Two checkers, both on the CPU:

* ``port``: liboracle.so, this repository's plain-C restatement of the
  reference evaluator (apsp_oracle.c, each function citing the reference
  lines it follows).
* ``ref``: the reference's own evaluator compiled from its sources into
  _ref/ by the recipe in Makefile (present only where the reference source
  tree was available at build time; the built files travel with the tree).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs use this package, and only to check or time against; the
product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_port = None
_ref_general = None
_ref_grid = None


def reference_source() -> Path | None:
    """The reference source tree: $GGB_REFERENCE, else the tree _ref/ was
    last built from (recorded in _ref/SOURCE by the Makefile), else None."""
    env = os.environ.get("GGB_REFERENCE")
    if env:
        return Path(env)
    rec = REF_DIR / "SOURCE"
    if rec.exists():
        p = rec.read_text().strip()
        if p:
            return Path(p)
    return None


def build(reference: str | os.PathLike | None = None) -> None:
    """Builds liboracle.so and, when a reference source tree is named
    (`reference`, else reference_source()) and exists, _ref/ from it."""
    src = Path(reference) if reference else reference_source()
    targets = ["oracle"]
    args = []
    if src is not None and src.exists():
        targets.append("ref")
        args.append(f"REF={src}")
    subprocess.run(["make", "-s", "-C", str(HERE), *args, *targets], check=True)


def port() -> C.CDLL:
    global _port
    if _port is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
        lib = C.CDLL(str(path))
        I, LL, P = C.c_int, C.c_longlong, C.c_void_p
        IP, DP, LP = C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_longlong)
        lib.oracle_general_eval.argtypes = [I, I, I, I, P, I, I, IP, DP, LP]
        lib.oracle_general_partial.argtypes = [I, I, I, I, P, I, I, I, I, IP, LP]
        lib.oracle_general_finish.argtypes = [I, I, LL, IP, DP]
        lib.oracle_grid_eval.argtypes = [I, I, I, P, I, P, IP, DP, LP]
        lib.oracle_grid_partial.argtypes = [I, I, I, P, I, P, I, I, IP, LP]
        lib.oracle_grid_finish.argtypes = [I, I, LL, IP, DP]
        lib.oracle_bfs_sums.argtypes = [I, I, P, P, I, IP, LP]
        lib.oracle_general_eval_nr.argtypes = [I, I, I, I, P, P, I, I, IP, DP, LP]
        lib.oracle_grid_eval_nr.argtypes = [I, I, P, I, P, I, P, IP, DP, LP]
        _port = lib
    return _port


def have_ref() -> bool:
    return (REF_DIR / "libref_general.so").exists() and (REF_DIR / "libref_grid.so").exists()


def have_ref_nr() -> bool:
    return (REF_DIR / "libref_general_nr.so").exists() and (REF_DIR / "libref_grid_nr.so").exists()


def _ref(kind: str) -> C.CDLL:
    global _ref_general, _ref_grid
    if kind == "general":
        if _ref_general is None:
            lib = C.CDLL(str(REF_DIR / "libref_general.so"))
            lib.evaluation.restype = C.c_bool
            lib.evaluation.argtypes = [C.c_int] * 5 + [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                                       C.c_int, C.c_int]
            lib.ref_set_ranks(0, 1)
            _ref_general = lib
        return _ref_general
    if _ref_grid is None:
        lib = C.CDLL(str(REF_DIR / "libref_grid.so"))
        lib.evaluation.restype = C.c_bool
        lib.evaluation.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_bool, C.c_void_p]
        lib.ref_set_ranks(0, 1)
        _ref_grid = lib
    return _ref_grid


def _adj(adj) -> np.ndarray:
    return np.ascontiguousarray(adj, dtype=np.int32)


def general(adj, based_nodes=None, groups=1, added_centers=0, algo=1):
    """Port: returns (connected, diameter, aspl, total)."""
    a = _adj(adj)
    n, d = a.shape
    if based_nodes is None:
        based_nodes = (n - added_centers) // groups
    dm, asp, tot = C.c_int(0), C.c_double(0.0), C.c_longlong(0)
    rc = port().oracle_general_eval(n, based_nodes, groups, d, a.ctypes.data, added_centers, algo,
                                    C.byref(dm), C.byref(asp), C.byref(tot))
    if rc < 0:
        raise ValueError(f"oracle_general_eval: {rc}")
    # the reference divides nothing for a disconnected graph: no total then
    return bool(rc), dm.value, asp.value, (tot.value if rc else 0)


def general_partial(adj, rank, procs, based_nodes=None, groups=1, added_centers=0, window_bits=0):
    """Port: rank's partial (diam, sum) before the MPI_Allreduce.  With
    window_bits (a multiple of 64) the source chunks are windows of that many
    sources instead of the reference's ceil(elements/procs) words, so that the
    partial can be compared with the GPU partial of the same window width."""
    a = _adj(adj)
    n, d = a.shape
    if based_nodes is None:
        based_nodes = (n - added_centers) // groups
    if window_bits % 64:
        raise ValueError("window_bits must be a multiple of 64")
    dm, sm = C.c_int(0), C.c_longlong(0)
    rc = port().oracle_general_partial(n, based_nodes, groups, d, a.ctypes.data, added_centers, window_bits // 64,
                                       rank, procs, C.byref(dm), C.byref(sm))
    if rc < 0:
        raise ValueError(f"oracle_general_partial: {rc}")
    return dm.value, sm.value


def grid(adj, rotate_hash, groups=1, based_nodes=None):
    """Port: returns (connected, diameter, aspl or None, total)."""
    a = _adj(adj)
    n, d = a.shape
    rh = np.ascontiguousarray(rotate_hash, dtype=np.int32)
    if based_nodes is None:
        based_nodes = n // groups
    dm, asp, tot = C.c_int(0), C.c_double(float("nan")), C.c_longlong(0)
    rc = port().oracle_grid_eval(n, d, groups, a.ctypes.data, based_nodes, rh.ctypes.data, C.byref(dm),
                                 C.byref(asp), C.byref(tot))
    if rc < 0:
        raise ValueError(f"oracle_grid_eval: {rc}")
    return bool(rc), dm.value, (asp.value if rc else None), (tot.value if rc else 0)


def bfs_sums(adj, n_sources=None, relabel=None):
    """Plain queue BFS: (max eccentricity or -1, Σ distances from the sources)."""
    a = _adj(adj)
    n, d = a.shape
    rh = None if relabel is None else np.ascontiguousarray(relabel, dtype=np.int32)
    e, s = C.c_int(0), C.c_longlong(0)
    port().oracle_bfs_sums(n, d, a.ctypes.data, None if rh is None else rh.ctypes.data,
                           n if n_sources is None else n_sources, C.byref(e), C.byref(s))
    return e.value, s.value


def ref_general(adj, based_nodes=None, groups=1, added_centers=0, algo=1, procs=1, rank=0):
    """Reference general evaluation() (compiled from its sources):
    returns (connected, diameter, aspl)."""
    lib = _ref("general")
    a = _adj(adj)
    n, d = a.shape
    if based_nodes is None:
        based_nodes = (n - added_centers) // groups
    lib.ref_set_ranks(rank, procs)
    dm, asp = C.c_int(0), C.c_double(0.0)
    ok = lib.evaluation(n, based_nodes, groups, n * d // 2, d, a.ctypes.data, C.byref(dm), C.byref(asp),
                        added_centers, algo)
    lib.ref_set_ranks(0, 1)
    return bool(ok), dm.value, asp.value


def ref_grid(adj, rotate_hash, groups=1, based_nodes=None, height=0, based_height=0, enable_bfs=False):
    """Reference grid evaluation(): returns (connected, diameter, aspl or None)."""
    lib = _ref("grid")
    a = _adj(adj)
    n, d = a.shape
    rh = np.ascontiguousarray(rotate_hash, dtype=np.int32)
    if based_nodes is None:
        based_nodes = n // groups
    dm, asp = C.c_int(0), C.c_double(float("nan"))
    ok = lib.evaluation(n, d, groups, a.ctypes.data, based_nodes, height, based_height, C.byref(dm),
                        C.byref(asp), bool(enable_bfs), rh.ctypes.data)
    return bool(ok), dm.value, (asp.value if ok else None)


def general_nr(adj, degs, based_nodes=None, groups=1, added_centers=0, algo=1):
    """Port, non-regular general: returns (connected, diameter, aspl, total)."""
    a = _adj(adj)
    n, d = a.shape
    nd = np.ascontiguousarray(degs, dtype=np.int32)
    if based_nodes is None:
        based_nodes = (n - added_centers) // groups
    dm, asp, tot = C.c_int(0), C.c_double(0.0), C.c_longlong(0)
    rc = port().oracle_general_eval_nr(n, based_nodes, groups, d, nd.ctypes.data, a.ctypes.data, added_centers,
                                       algo, C.byref(dm), C.byref(asp), C.byref(tot))
    if rc < 0:
        raise ValueError(f"oracle_general_eval_nr: {rc}")
    return bool(rc), dm.value, asp.value, (tot.value if rc else 0)


def grid_nr(adj, degs, rotate_hash, groups=1, based_nodes=None):
    """Port, non-regular grid: returns (connected, diameter, aspl or None, total)."""
    a = _adj(adj)
    n, d = a.shape
    nd = np.ascontiguousarray(degs, dtype=np.int32)
    rh = np.ascontiguousarray(rotate_hash, dtype=np.int32)
    if based_nodes is None:
        based_nodes = n // groups
    dm, asp, tot = C.c_int(0), C.c_double(float("nan")), C.c_longlong(0)
    rc = port().oracle_grid_eval_nr(n, d, nd.ctypes.data, groups, a.ctypes.data, based_nodes, rh.ctypes.data,
                                    C.byref(dm), C.byref(asp), C.byref(tot))
    if rc < 0:
        raise ValueError(f"oracle_grid_eval_nr: {rc}")
    return bool(rc), dm.value, (asp.value if rc else None), (tot.value if rc else 0)


_ref_nr = {}


def ref_general_nr(adj, degs, based_nodes=None, groups=1, added_centers=0, algo=1):
    """The reference's non-regular general evaluation(): (connected, diameter, aspl)."""
    if "g" not in _ref_nr:
        lib = C.CDLL(str(REF_DIR / "libref_general_nr.so"))
        lib.evaluation.restype = C.c_bool
        lib.evaluation.argtypes = [C.c_int] * 5 + [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int,
                                                   C.c_void_p, C.c_int]
        lib.ref_set_ranks(0, 1)
        _ref_nr["g"] = lib
    lib = _ref_nr["g"]
    a = _adj(adj)
    n, d = a.shape
    nd = np.ascontiguousarray(degs, dtype=np.int32)
    if based_nodes is None:
        based_nodes = (n - added_centers) // groups
    dm, asp = C.c_int(0), C.c_double(0.0)
    ok = lib.evaluation(n, based_nodes, groups, int(nd.sum()) // 2, d, a.ctypes.data, C.byref(dm), C.byref(asp),
                        added_centers, nd.ctypes.data, algo)
    return bool(ok), dm.value, asp.value


def ref_grid_nr(adj, degs, rotate_hash, groups=1, based_nodes=None):
    """The reference's non-regular grid evaluation(): (connected, diameter, aspl or None)."""
    if "r" not in _ref_nr:
        lib = C.CDLL(str(REF_DIR / "libref_grid_nr.so"))
        lib.evaluation.restype = C.c_bool
        lib.evaluation.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_bool, C.c_void_p]
        lib.ref_set_ranks(0, 1)
        _ref_nr["r"] = lib
    lib = _ref_nr["r"]
    a = _adj(adj)
    n, d = a.shape
    nd = np.ascontiguousarray(degs, dtype=np.int32)
    rh = np.ascontiguousarray(rotate_hash, dtype=np.int32)
    if based_nodes is None:
        based_nodes = n // groups
    dm, asp = C.c_int(0), C.c_double(float("nan"))
    ok = lib.evaluation(n, d, nd.ctypes.data, groups, a.ctypes.data, based_nodes, 0, 0, C.byref(dm), C.byref(asp),
                        False, rh.ctypes.data)
    return bool(ok), dm.value, (asp.value if ok else None)



def level_stats(adj, levels: int = 32) -> np.ndarray:
    """[n][levels]: entry [v][k] = vertices not within distance k of v, by a
    plain BFS from every vertex (the per-vertex statistics the profile
    kernel accumulates; unreachable vertices count at every level)."""
    a = np.asarray(adj)
    n = a.shape[0]
    out = np.zeros((n, levels), dtype=np.int64)
    for s in range(n):
        dist = np.full(n, -1, dtype=np.int64)
        dist[s] = 0
        frontier = [s]
        k = 0
        while frontier:
            k += 1
            nxt = []
            for u in frontier:
                for w in a[u]:
                    if dist[w] < 0:
                        dist[w] = k
                        nxt.append(int(w))
            frontier = nxt
        for q in range(levels):
            out[s, q] = int(np.sum((dist < 0) | (dist > q)))
    return out
