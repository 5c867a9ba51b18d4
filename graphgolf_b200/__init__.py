"""graphgolf_b200 -- B200-native exact APSP evaluator for GraphGolf graphs.

The hot path is the bit-parallel all-pairs BFS that the reference's
simulated annealing calls once per step (general/evaluation.c:153-263,
grid/evaluation.c:122-190), rebuilt as a persistent sm_100a CUDA kernel
behind the reference's own C ``evaluation()`` interface.
"""
from ._native import NativeLibraryMissing, load
from .anneal import Annealer, FilterNet, checkpoint_graph
from .batch import Batch
from .evaluator import (BFS, MATRIX_OP, MATRIX_OP_MEM_SAVING, EvaluationError, Result, evaluate,
                        evaluate_grid, evaluate_grid_nonregular, evaluate_nonregular, evaluate_partial, evaluation, finish_general, grid_evaluation,
                        kernel_launches, set_ball, set_tuning)

__all__ = [
    "Annealer", "BFS", "Batch", "FilterNet", "MATRIX_OP", "MATRIX_OP_MEM_SAVING", "EvaluationError", "NativeLibraryMissing", "Result",
    "evaluate", "evaluate_grid", "evaluate_grid_nonregular", "evaluate_nonregular", "evaluate_partial", "evaluation", "finish_general", "grid_evaluation",
    "checkpoint_graph", "kernel_launches", "load", "set_ball", "set_tuning",
]
