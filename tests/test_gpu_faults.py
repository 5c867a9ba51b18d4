"""Failure paths of the CUDA evaluator.  Nothing here faults or hangs a GPU:
bad inputs are caught by the kernels' own bounds checks and reported as
status codes, and the barrier test makes a bounded wait run out (a phantom
arrival that nothing provides) so the kernel returns an error itself."""
import numpy as np
import pytest

import graphgolf_b200 as gg
import oracle
from graphgolf_b200 import graphs

pytestmark = pytest.mark.gpu


def _ok_after(lib):
    adj = graphs.random_regular(500, 6, 3).adj
    r = gg.evaluate(adj)
    assert (r.connected, r.diameter, r.aspl, r.total) == oracle.general(adj)


def test_adjacency_out_of_range(gpu):
    adj = graphs.random_regular(400, 6, 4).adj.copy()
    adj[123, 2] = 400
    with pytest.raises(gg.EvaluationError) as e:
        gg.evaluate(adj)
    assert e.value.code == -3
    adj[123, 2] = -7
    with pytest.raises(gg.EvaluationError) as e:
        gg.evaluate(adj)
    assert e.value.code == -3
    _ok_after(gpu)


def test_rotate_hash_not_a_permutation(gpu):
    gr = graphs.grid_regular(10, 10, 4, 3, 1)
    rh = np.arange(100, dtype=np.int32)
    rh[5] = 6
    with pytest.raises(gg.EvaluationError) as e:
        gg.evaluate_grid(gr.adj, rh)
    assert e.value.code == -5
    rh[5] = 100
    with pytest.raises(gg.EvaluationError) as e:
        gg.evaluate_grid(gr.adj, rh)
    assert e.value.code == -5
    _ok_after(gpu)


def test_invalid_sizes(gpu):
    adj = graphs.random_regular(100, 4, 5).adj
    with pytest.raises(gg.EvaluationError) as e:
        gg.evaluation(100, 30, 3, 200, 4, adj)      # 30*3 != 100
    assert e.value.code == -1
    with pytest.raises(gg.EvaluationError):
        gg.evaluation(100, 100, 1, 200, 5, adj)     # wrong degree for the array
    _ok_after(gpu)


def test_barrier_wait_runs_out(gpu):
    """A barrier that waits for one arrival too many must give up after its
    time limit on every CTA, report GGB_ETIMEOUT, and leave the context usable."""
    lib = gg.load()
    adj = graphs.random_regular(2000, 6, 6).adj
    assert lib.ggb_set_barrier_test(2_000_000, 1) == 0     # 2 ms limit, one phantom arrival
    try:
        with pytest.raises(gg.EvaluationError) as e:
            gg.evaluate(adj)
        assert e.value.code == -4
    finally:
        assert lib.ggb_set_barrier_test(2_000_000_000, 0) == 0
    _ok_after(gpu)
