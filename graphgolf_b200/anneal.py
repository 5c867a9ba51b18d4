"""Simulated annealing with the whole step on the device, and its learned
proposal filter.

``Annealer`` wraps the ``ggb_sa_*`` C ABI (include/graphgolf_b200.h): every
step draws 2-opt swaps of the current graph, optionally ranks them with the
filter network, evaluates the best ones exactly in one batch launch, composes
the disjoint improving ones into one more exactly evaluated graph and accepts
by the reference's rule (general/sa.c:371-411).  ``candidates=1`` without
composition is the reference's plain step (general/sa.c:413-520) on the
device.  ``FilterNet`` exposes the filter's network (ggb_mlp_*) on its own.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import ggb_sa_stats, load
from .evaluator import _raise
from .graphs import Graph


@dataclass(frozen=True)
class Stats:
    step: int
    accepts: int
    multi_accepts: int
    moved_swaps: int
    evals: int
    pred_accepts: int
    unevaluated: int
    cur_diam: int
    best_diam: int
    cur_total: int
    best_total: int
    cur_aspl: float
    best_aspl: float
    temp: float
    done: bool
    delta: bool         # candidates evaluated against the kept base (else in full)


class Annealer:
    """Device annealing of `g`.  With g.groups > 1 (edges in the reference's
    symmetric line order) every move is an orbit move that keeps the symmetry
    and there is no proposal filter; grid graphs add a length limit with
    ``grid()``."""

    def __init__(self, g: Graph, candidates: int = 1, proposals: int | None = None, compose: int = 0,
                 seed: int = 1):
        self._lib = load()
        self.nodes, self.degree, self.lines, self.groups = g.nodes, g.degree, g.lines, g.groups
        self.candidates = candidates
        e = np.ascontiguousarray(g.edges, dtype=np.int32)
        h = C.c_void_p()
        if g.groups > 1:
            if proposals not in (None, candidates):
                raise ValueError("graphs with symmetry groups are annealed without a proposal filter")
            _raise(self._lib.ggb_sa_create_symmetric(g.nodes, g.degree, g.groups, e.ctypes.data, candidates,
                                                     compose, seed, C.byref(h)))
        else:
            _raise(self._lib.ggb_sa_create(g.nodes, g.degree, e.ctypes.data, candidates,
                                           proposals if proposals else candidates, compose, seed, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ggb_sa_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "Annealer":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def schedule(self, temp: float = 0.0, cooling: float = 1.0, hill_climbing: bool = True) -> None:
        _raise(self._lib.ggb_sa_set_schedule(self._h, temp, cooling, 1 if hill_climbing else 0))

    def grid(self, height: int, max_length: int) -> None:
        """Grid graph: vertex v = (v // height, v % height); every move keeps
        both new edges within Manhattan length max_length (grid/sa.c:137-221)."""
        _raise(self._lib.ggb_sa_set_grid(self._h, height, max_length))

    def predicted(self, composites: int = 4, max_swaps: int = 64) -> None:
        """Predicted composites per step (filter only) and the largest's size."""
        _raise(self._lib.ggb_sa_set_predicted(self._h, composites, max_swaps))

    def target(self, diameter: int, total: int) -> None:
        _raise(self._lib.ggb_sa_set_target(self._h, diameter, total))

    def autotune(self, iters: int = 1) -> tuple[int, int, float]:
        w, t, ms = C.c_int(), C.c_int(), C.c_double()
        _raise(self._lib.ggb_sa_autotune(self._h, iters, C.byref(w), C.byref(t), C.byref(ms)))
        return w.value, t.value, ms.value

    def run(self, steps: int) -> Stats:
        st = ggb_sa_stats()
        _raise(self._lib.ggb_sa_run(self._h, steps, C.byref(st)))
        return Stats(st.step, st.accepts, st.multi_accepts, st.moved_swaps, st.evals, st.pred_accepts,
                     st.unevaluated, st.cur_diam, st.best_diam,
                     st.cur_total, st.best_total, st.cur_aspl, st.best_aspl, st.temp, bool(st.done),
                     bool(st.delta))

    def edges(self, best: bool = False) -> np.ndarray:
        out = np.empty((self.lines, 2), dtype=np.int32)
        _raise(self._lib.ggb_sa_edges(self._h, 1 if best else 0, out.ctypes.data))
        return out

    def last_step(self) -> tuple[np.ndarray, np.ndarray]:
        """(predicted, exact label) of the last step's evaluated candidates."""
        k = self.candidates
        pr = np.empty(k, dtype=np.float32)
        lb = np.empty(k, dtype=np.float32)
        _raise(self._lib.ggb_sa_last_step(self._h, pr.ctypes.data, lb.ctypes.data))
        return pr, lb

    def check_delta(self, with_dense: bool = False):
        """(compared, mismatches, unevaluated[, dense windows]): fresh
        candidates evaluated against the base and in full."""
        c, m, u, dn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _raise(self._lib.ggb_sa_check_delta(self._h, C.byref(c), C.byref(m), C.byref(u), C.byref(dn)))
        return (c.value, m.value, u.value, dn.value) if with_dense else (c.value, m.value, u.value)

    def base_plan(self) -> tuple[int, int]:
        """(CTAs per team, teams) of the kept base's build, (0, 0) without one."""
        t, n = C.c_int(), C.c_int()
        _raise(self._lib.ggb_sa_base_plan(self._h, C.byref(t), C.byref(n)))
        return t.value, n.value

    def save(self) -> bytes:
        """A checkpoint of the run: graph, best graph, step, schedule,
        counters and (with a filter) the network's training state."""
        n = int(self._lib.ggb_sa_checkpoint_bytes(self._h))
        buf = C.create_string_buffer(n)
        _raise(self._lib.ggb_sa_save(self._h, buf, n))
        return buf.raw

    def restore(self, ckpt: bytes) -> None:
        """Continues the run saved in `ckpt`.  The annealer must have been
        created from ``checkpoint_graph(ckpt)`` with the same arguments."""
        _raise(self._lib.ggb_sa_restore(self._h, ckpt, len(ckpt)))

    def profile(self) -> np.ndarray:
        """[nodes][32]: entry [v][k] = vertices farther than k from v."""
        out = np.empty((self.nodes, 32), dtype=np.uint32)
        _raise(self._lib.ggb_sa_profile(self._h, out.ctypes.data))
        return out


def checkpoint_graph(ckpt: bytes, best: bool = False) -> Graph:
    """The current (or best) graph of an annealing checkpoint, to create the
    annealer that ``Annealer.restore`` continues."""
    from .graphs import create_adj
    lib = load()
    n, d, g, lines = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    _raise(lib.ggb_sa_checkpoint_info(ckpt, len(ckpt), C.byref(n), C.byref(d), C.byref(g), C.byref(lines)))
    e = np.empty((lines.value, 2), dtype=np.int32)
    _raise(lib.ggb_sa_checkpoint_edges(ckpt, len(ckpt), 1 if best else 0, e.ctypes.data))
    return Graph(n.value, d.value, e, create_adj(n.value, d.value, e), groups=g.value)


class FilterNet:
    """The proposal filter's network: 32 -> 256 -> 256 -> 1 ReLU MLP, BF16
    tensor cores with FP32 accumulation, Adam on the mean squared error."""

    FEATURES, HIDDEN = 32, 256

    def __init__(self, max_rows: int = 4096, seed: int = 1):
        self._lib = load()
        h = C.c_void_p()
        _raise(self._lib.ggb_mlp_create(max_rows, seed, C.byref(h)))
        self._h = h
        self.n_params = int(self._lib.ggb_mlp_param_count())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ggb_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, dtype=np.float32)
        _raise(self._lib.ggb_mlp_get_params(self._h, p.ctypes.data))
        return p

    @params.setter
    def params(self, p) -> None:
        a = np.ascontiguousarray(p, dtype=np.float32)
        if a.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters")
        _raise(self._lib.ggb_mlp_set_params(self._h, a.ctypes.data))

    def set_adam(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        _raise(self._lib.ggb_mlp_set_adam(self._h, lr, beta1, beta2, eps))

    def forward(self, x) -> np.ndarray:
        a = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty(a.shape[0], dtype=np.float32)
        _raise(self._lib.ggb_mlp_forward_host(self._h, a.ctypes.data, a.shape[0], y.ctypes.data))
        return y

    def time_forward(self, x, reps: int = 50) -> float:
        """Mean device time (ms) of one inference forward over the rows of x,
        timed with CUDA events over `reps` back-to-back launches."""
        a = np.ascontiguousarray(x, dtype=np.float32)
        ms = C.c_double()
        _raise(self._lib.ggb_mlp_time_forward(self._h, a.ctypes.data, a.shape[0], reps, C.byref(ms)))
        return ms.value

    def grads(self, x, t) -> tuple[float, np.ndarray]:
        a = np.ascontiguousarray(x, dtype=np.float32)
        b = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_float()
        _raise(self._lib.ggb_mlp_grads_host(self._h, a.ctypes.data, b.ctypes.data, a.shape[0], C.byref(loss),
                                            g.ctypes.data))
        return loss.value, g

    def train(self, x, t, steps: int) -> float:
        a = np.ascontiguousarray(x, dtype=np.float32)
        b = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        _raise(self._lib.ggb_mlp_train_host(self._h, a.ctypes.data, b.ctypes.data, a.shape[0], steps,
                                            C.byref(loss)))
        return loss.value
