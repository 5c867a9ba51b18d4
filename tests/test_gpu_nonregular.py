"""The non-regular evaluators (the reference's variants/not_regular_general_graph
and variants/not_regular_grid_graph) on the GPU against the oracle: rows hold
num_degrees[i] neighbours; the unused slots are ignored in the based phase
and read, as the reference reads them, in the added-centre phase."""
import numpy as np
import pytest

import graphgolf_b200 as gg
import oracle
from graphgolf_b200 import graphs
from _cases import union_graph  # noqa: F401  (shared helpers)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ball", [-1, 0, 1])
@pytest.mark.parametrize("n,d,drop,g,ac", [(300, 6, 150, 1, 0), (512, 8, 300, 4, 0), (610, 5, 100, 2, 10),
                                           (3000, 12, 4000, 1, 0), (2050, 16, 3000, 8, 2), (6000, 7, 9000, 1, 0)])
def test_general_nonregular(gpu, ball, n, d, drop, g, ac):
    gr = graphs.random_regular(n, d, n + drop)
    _, adj, deg = graphs.nonregular(gr, drop, 7)
    bn = (n - ac) // g
    want = oracle.general_nr(adj, deg, based_nodes=bn, groups=g, added_centers=ac)
    try:
        gg.set_ball(ball)
        r = gg.evaluate_nonregular(adj, deg, based_nodes=bn, groups=g, added_centers=ac)
    finally:
        gg.set_ball(-1)
    assert (r.connected, r.diameter, r.aspl, r.total) == want


def test_general_nonregular_padding_ignored(gpu):
    """Without added centres the padding is never read: -1 there is fine."""
    gr = graphs.random_regular(800, 8, 11)
    _, adj, deg = graphs.nonregular(gr, 500, 5, pad=-1)
    adj = adj.copy()
    for i in range(adj.shape[0]):
        adj[i, deg[i]:] = -1
    want = oracle.general_nr(adj, deg)
    r = gg.evaluate_nonregular(adj, deg)
    assert (r.connected, r.diameter, r.aspl, r.total) == want
    # with added centres the whole row is read, as by the reference: -1 is an invalid vertex
    with pytest.raises(gg.EvaluationError) as e:
        gg.evaluate_nonregular(adj, deg, based_nodes=780, added_centers=20)
    assert e.value.code == -3


def test_general_nonregular_bad_degree(gpu):
    gr = graphs.random_regular(100, 4, 1)
    deg = np.full(100, 4, dtype=np.int32)
    deg[7] = 5
    with pytest.raises(gg.EvaluationError) as e:
        gg.evaluate_nonregular(gr.adj, deg)
    assert e.value.code == -1


def test_regular_as_nonregular(gpu):
    gr = graphs.random_regular(2000, 10, 3)
    r1 = gg.evaluate(gr.adj)
    r2 = gg.evaluate_nonregular(gr.adj, np.full(2000, 10, dtype=np.int32))
    assert (r1.connected, r1.diameter, r1.aspl, r1.total) == (r2.connected, r2.diameter, r2.aspl, r2.total)


@pytest.mark.parametrize("w,h,d,drop,g", [(16, 16, 6, 100, 1), (20, 20, 4, 60, 2), (18, 18, 6, 120, 4),
                                          (60, 60, 6, 2000, 1)])
def test_grid_nonregular(gpu, w, h, d, drop, g):
    gr = graphs.grid_regular(w, h, d, 3, w + drop)
    _, adj, deg = graphs.nonregular(gr, drop, 3)
    rh = graphs.rotate_hash(gr.nodes, h, w, g)
    want = oracle.grid_nr(adj, deg, rh, groups=g)
    r = gg.evaluate_grid_nonregular(adj, deg, rh, groups=g)
    assert (r.connected, r.diameter, r.total) == (want[0], want[1], want[3])
    if r.connected:
        assert r.aspl == want[2]
