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
    good = adj[123, 2]
    # 400 and 65535 travel as 16-bit ids; the others make the upload fall back
    # to plain ints.  Each is caught by the device bounds check, and the next
    # upload of the valid graph is exact.
    for bad in (400, -7, 65535, 65536, 70000, 1 << 30, -65536):
        adj[123, 2] = bad
        with pytest.raises(gg.EvaluationError) as e:
            gg.evaluate(adj)
        assert e.value.code == -3, bad
        adj[123, 2] = good
        r = gg.evaluate(adj)
        assert (r.connected, r.diameter, r.aspl, r.total) == oracle.general(adj), bad


def test_out_of_range_id_in_a_later_staging_unit(gpu):
    """An upload of several staging units (N=40000, d=8: 320 000 ids) with
    one id past 16 bits in the last unit: the narrowed units already sent are
    dropped, the ints are sent as they are, and the device reports the id."""
    adj = graphs.random_regular(40000, 8, 9).adj.copy()
    r0 = gg.evaluate(adj)
    assert (r0.connected, r0.diameter, r0.aspl, r0.total) == oracle.general(adj)
    good = adj[39990, 5]
    for bad in (40000, 65536, -2):
        adj[39990, 5] = bad
        with pytest.raises(gg.EvaluationError) as e:
            gg.evaluate(adj)
        assert e.value.code == -3, bad
        adj[39990, 5] = good
        r = gg.evaluate(adj)
        assert (r.connected, r.diameter, r.aspl, r.total) == (r0.connected, r0.diameter, r0.aspl, r0.total)


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
