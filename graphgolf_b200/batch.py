"""Batched exact APSP: many general graphs, of uneven sizes, in one launch.

``Batch`` wraps the ``ggb_batch_*`` C ABI (include/graphgolf_b200.h).  The
graphs' sizes are fixed at creation; their adjacency arrays can be replaced
from the host (``evaluate``) or written in place on the device (``adj_ptr``),
and every launch is one replay of a CUDA graph.  Each graph's ``Result`` is
the one ``evaluate`` gives that graph alone.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from ._native import ggb_result, load
from .evaluator import EvaluationError, Result, _raise


class Batch:
    def __init__(self, nodes: Sequence[int], degree: Sequence[int] | int, groups: Sequence[int] | int = 1):
        n = len(nodes)
        if n == 0:
            raise EvaluationError(-1, "a batch needs at least one graph")
        self.nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        self.degree = np.ascontiguousarray(np.broadcast_to(degree, (n,)), dtype=np.int32)
        self.groups = np.ascontiguousarray(np.broadcast_to(groups, (n,)), dtype=np.int32)
        if np.any(self.nodes % self.groups):
            raise EvaluationError(-1, "every graph's nodes must be a multiple of its groups")
        self.based = np.ascontiguousarray(self.nodes // self.groups, dtype=np.int32)
        self._lib = load()
        h = C.c_void_p()
        _raise(self._lib.ggb_batch_create(n, self.nodes.ctypes.data, self.based.ctypes.data, self.groups.ctypes.data,
                                          self.degree.ctypes.data, C.byref(h)))
        self._h = h
        self._res = (ggb_result * n)()

    def __len__(self) -> int:
        return len(self.nodes)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ggb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "Batch":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    # ---- plan ------------------------------------------------------------
    def set_plan(self, window_bits: int = 0, team_ctas: int = 0) -> None:
        _raise(self._lib.ggb_batch_set_plan(self._h, window_bits, team_ctas))

    @property
    def plan(self) -> tuple[int, int, int]:
        """(window_bits, team_ctas, teams)."""
        w, t, k = C.c_int(), C.c_int(), C.c_int()
        _raise(self._lib.ggb_batch_get_plan(self._h, C.byref(w), C.byref(t), C.byref(k)))
        return w.value, t.value, k.value

    def autotune(self, iters: int = 2) -> tuple[int, int, float]:
        """Times every feasible plan on the current adjacency; keeps and
        returns the fastest (window_bits, team_ctas, ms)."""
        w, t, ms = C.c_int(), C.c_int(), C.c_double()
        _raise(self._lib.ggb_batch_autotune(self._h, iters, C.byref(w), C.byref(t), C.byref(ms)))
        return w.value, t.value, ms.value

    # ---- data ------------------------------------------------------------
    def adj_ptr(self, i: int) -> int:
        """Device address of graph i's [nodes][degree] int32 adjacency."""
        p = C.c_void_p()
        _raise(self._lib.ggb_batch_adj_device(self._h, i, C.byref(p)))
        return int(p.value)

    def adj_view(self, i: int):
        """A torch int32 CUDA tensor [nodes][degree] aliasing graph i's
        adjacency inside the batch (writes go straight to the batch)."""
        import torch
        n, d = int(self.nodes[i]), int(self.degree[i])
        ptr = self.adj_ptr(i)

        class _DeviceArray:
            __cuda_array_interface__ = {"shape": (n, d), "typestr": "<i4", "data": (ptr, False), "version": 2,
                                        "strides": None}

        return torch.as_tensor(_DeviceArray(), device="cuda")

    def _ptrs(self, adjs) -> tuple[list[np.ndarray], C.Array]:
        if len(adjs) != len(self):
            raise EvaluationError(-1, f"{len(adjs)} adjacency arrays for a batch of {len(self)}")
        keep = []
        for i, a in enumerate(adjs):
            arr = np.ascontiguousarray(a, dtype=np.int32)
            if arr.size != int(self.nodes[i]) * int(self.degree[i]):
                raise EvaluationError(-1, f"graph {i}: adjacency has {arr.size} entries, expected "
                                          f"{int(self.nodes[i]) * int(self.degree[i])}")
            keep.append(arr)
        ptrs = (C.c_void_p * len(keep))(*[k.ctypes.data for k in keep])
        return keep, ptrs

    def upload(self, adjs, stream: int | None = None) -> None:
        keep, ptrs = self._ptrs(adjs)
        _raise(self._lib.ggb_batch_upload(self._h, ptrs, stream))
        del keep

    # ---- evaluation ------------------------------------------------------
    def launch(self, stream: int | None = None) -> None:
        _raise(self._lib.ggb_batch_launch(self._h, stream))

    def collect(self, stream: int | None = None) -> list[Result]:
        _raise(self._lib.ggb_batch_collect(self._h, stream, self._res))
        return [Result.from_c(r) for r in self._res]

    def evaluate(self, adjs) -> list[Result]:
        """Upload + one launch + results, from host arrays."""
        keep, ptrs = self._ptrs(adjs)
        _raise(self._lib.ggb_batch_eval(self._h, ptrs, self._res))
        del keep
        return [Result.from_c(r) for r in self._res]

    def kernel_ms(self) -> float:
        ms = C.c_double()
        _raise(self._lib.ggb_batch_kernel_ms(self._h, C.byref(ms)))
        return ms.value
