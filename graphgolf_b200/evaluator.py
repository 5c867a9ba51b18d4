"""Python face of the B200 exact APSP evaluator.

``evaluation`` and ``grid_evaluation`` mirror the reference's C functions
(general/common.h:112-113, grid/common.h:88-90): same argument meaning, same
return value and written values.  Where the reference aborts through ERROR()
(general/common.h:67-70), these raise ``EvaluationError``.  ``evaluate`` and
``evaluate_grid`` return the full ``Result`` (exact integer total, levels).

Everything runs in libgraphgolf_b200.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from ._native import ggb_partial, ggb_result, last_error, load

BFS, MATRIX_OP, MATRIX_OP_MEM_SAVING = 0, 1, 2   # general/common.h:58-60

STATUS = {0: "ok", -1: "EINVAL", -2: "ECUDA", -3: "EADJ", -4: "ETIMEOUT", -5: "EPERM", -6: "ENOMEM"}


class EvaluationError(RuntimeError):
    """The evaluator rejected its input or the device failed."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


@dataclass(frozen=True)
class Result:
    connected: bool
    diameter: int
    aspl: float
    total: int          # exact Σ d(u,v) over ordered pairs, group-weighted
    levels: int         # BFS levels executed over all source windows
    windows: int
    window_bits: int
    dense_levels: int   # of which dense OR-gather sweeps

    @staticmethod
    def from_c(r: ggb_result) -> "Result":
        return Result(bool(r.connected), int(r.diameter), float(r.aspl), int(r.total), int(r.levels),
                      int(r.windows), int(r.window_bits), int(r.dense_levels))


def _raise(rc: int) -> None:
    if rc != 0:
        raise EvaluationError(rc, last_error())


def _adj_array(adj, nodes: int, degree: int) -> np.ndarray:
    a = np.ascontiguousarray(adj, dtype=np.int32)
    if a.size != nodes * degree:
        raise EvaluationError(-1, f"adjacency has {a.size} entries, expected nodes*degree = {nodes * degree}")
    return a


def evaluate(adj, based_nodes: int | None = None, groups: int = 1, added_centers: int = 0) -> Result:
    """Exact APSP of a general graph given its [nodes][degree] adjacency."""
    a = np.ascontiguousarray(adj, dtype=np.int32)
    if a.ndim != 2:
        raise EvaluationError(-1, "adjacency must be a 2-D [nodes][degree] array")
    nodes, degree = a.shape
    if based_nodes is None:
        based_nodes = (nodes - added_centers) // groups
    r = ggb_result()
    _raise(load().ggb_eval_general(nodes, based_nodes, groups, degree, a.ctypes.data, added_centers, C.byref(r)))
    return Result.from_c(r)


def evaluate_grid(adj, rotate_hash, groups: int = 1, based_nodes: int | None = None) -> Result:
    a = np.ascontiguousarray(adj, dtype=np.int32)
    nodes, degree = a.shape
    rh = np.ascontiguousarray(rotate_hash, dtype=np.int32)
    if rh.shape != (nodes,):
        raise EvaluationError(-1, "rotate_hash must have one entry per vertex")
    if based_nodes is None:
        based_nodes = nodes // groups
    r = ggb_result()
    _raise(load().ggb_eval_grid(nodes, degree, groups, a.ctypes.data, based_nodes, rh.ctypes.data, C.byref(r)))
    return Result.from_c(r)


def evaluate_nonregular(adj, num_degrees, based_nodes: int | None = None, groups: int = 1,
                        added_centers: int = 0) -> Result:
    """Exact APSP of a non-regular general graph: row i of the
    [nodes][max_degree] adjacency holds num_degrees[i] neighbours
    (variants/not_regular_general_graph/evaluation.c:378-393)."""
    a = np.ascontiguousarray(adj, dtype=np.int32)
    nodes, max_degree = a.shape
    nd = np.ascontiguousarray(num_degrees, dtype=np.int32)
    if nd.shape != (nodes,):
        raise EvaluationError(-1, "num_degrees must have one entry per vertex")
    if based_nodes is None:
        based_nodes = (nodes - added_centers) // groups
    r = ggb_result()
    _raise(load().ggb_eval_general_nonregular(nodes, based_nodes, groups, max_degree, nd.ctypes.data,
                                              a.ctypes.data, added_centers, C.byref(r)))
    return Result.from_c(r)


def evaluate_grid_nonregular(adj, degree, rotate_hash, groups: int = 1, based_nodes: int | None = None) -> Result:
    """Exact APSP of a non-regular grid graph (variants/not_regular_grid_graph/
    evaluation.c:192-207): row i holds degree[i] neighbours."""
    a = np.ascontiguousarray(adj, dtype=np.int32)
    nodes, max_degree = a.shape
    dg = np.ascontiguousarray(degree, dtype=np.int32)
    rh = np.ascontiguousarray(rotate_hash, dtype=np.int32)
    if dg.shape != (nodes,) or rh.shape != (nodes,):
        raise EvaluationError(-1, "degree and rotate_hash must have one entry per vertex")
    if based_nodes is None:
        based_nodes = nodes // groups
    r = ggb_result()
    _raise(load().ggb_eval_grid_nonregular(nodes, max_degree, dg.ctypes.data, groups, a.ctypes.data, based_nodes,
                                           rh.ctypes.data, C.byref(r)))
    return Result.from_c(r)


def evaluation(nodes: int, based_nodes: int, groups: int, lines: int, degree: int, adj,
               added_centers: int = 0, algo: int = MATRIX_OP) -> tuple[bool, int, float]:
    """general evaluation(): returns (connected, diameter, ASPL) as the C
    function returns/writes them (INT_MAX / DBL_MAX when disconnected)."""
    a = _adj_array(adj, nodes, degree)
    r = ggb_result()
    _raise(load().ggb_eval_general(nodes, based_nodes, groups, degree, a.ctypes.data, added_centers, C.byref(r)))
    return bool(r.connected), int(r.diameter), float(r.aspl)


def grid_evaluation(nodes: int, degree: int, groups: int, adjacency, based_nodes: int, height: int,
                    based_height: int, enable_bfs: bool, rotate_hash,
                    aspl_in: float = math.nan) -> tuple[bool, int, float]:
    """grid evaluation(): returns (connected, diameter, ASPL).  ASPL is
    ``aspl_in`` (the caller's previous value) when disconnected, as the C
    function leaves it untouched."""
    a = _adj_array(adjacency, nodes, degree)
    rh = np.ascontiguousarray(rotate_hash, dtype=np.int32)
    r = ggb_result()
    _raise(load().ggb_eval_grid(nodes, degree, groups, a.ctypes.data, based_nodes, rh.ctypes.data, C.byref(r)))
    return bool(r.connected), int(r.diameter), (float(r.aspl) if r.connected else aspl_in)


def evaluate_partial(adj, rank: int, procs: int, based_nodes: int | None = None, groups: int = 1,
                     added_centers: int = 0) -> ggb_partial:
    """This rank's share of the source windows (general/evaluation.c:166)."""
    a = np.ascontiguousarray(adj, dtype=np.int32)
    nodes, degree = a.shape
    if based_nodes is None:
        based_nodes = (nodes - added_centers) // groups
    p = ggb_partial()
    _raise(load().ggb_eval_general_partial(nodes, based_nodes, groups, degree, a.ctypes.data, added_centers,
                                           rank, procs, C.byref(p)))
    return p


def finish_general(nodes: int, diam: int, disconnected: int, total_sum: int) -> Result:
    """Completes all-reduced partials (MAX diam, MAX disconnected, SUM sum)."""
    p = ggb_partial(diam, disconnected, total_sum, 0, 0, 0, 0)
    r = ggb_result()
    _raise(load().ggb_finish_general(nodes, C.byref(p), C.byref(r)))
    return Result.from_c(r)


def set_tuning(window_bits: int = 0, ctas: int = 0) -> None:
    """Forces the source-window width / grid size (0 = automatic)."""
    _raise(load().ggb_set_tuning(window_bits, ctas))


def set_ball(mode: int = -1) -> None:
    """Ball pre-pass policy: -1 automatic, 0 never, 1 whenever feasible."""
    _raise(load().ggb_set_ball(mode))


def kernel_launches() -> int:
    return int(load().ggb_kernel_launches())
