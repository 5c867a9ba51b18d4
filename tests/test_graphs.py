"""Host-side graph utilities the batch and annealing paths rely on (CPU)."""
import numpy as np

from graphgolf_b200 import graphs


def test_swap_2opt_valid_and_minimal():
    g = graphs.random_regular(500, 6, 3)
    h = graphs.swap_2opt(g, 11)
    assert graphs.verify(h) == 0
    changed = np.any(g.edges != h.edges, axis=1)
    assert changed.sum() == 2
    # the four endpoints of the two changed lines are the same vertices
    a = sorted(g.edges[changed].ravel().tolist())
    b = sorted(h.edges[changed].ravel().tolist())
    assert a == b
    # the degree sequence is unchanged and every row is the create_adj of the edges
    assert np.array_equal(h.adj, graphs.create_adj(h.nodes, h.degree, h.edges))


def test_swap_2opt_deterministic():
    g = graphs.random_regular(300, 4, 1)
    assert np.array_equal(graphs.swap_2opt(g, 5).edges, graphs.swap_2opt(g, 5).edges)
    assert not np.array_equal(graphs.swap_2opt(g, 5).edges, graphs.swap_2opt(g, 6).edges)


def test_batch_workload_shape():
    w = graphs.batch_workload(candidates=12, degree=12, n_lo=512, n_hi=16384, base_nodes=4096, seed=3)
    assert len(w) == 13 and w[0].nodes == 4096
    assert all(512 <= x.nodes <= 16384 + 1 for x in w[1:])
    assert all(graphs.verify(x) == 0 for x in w)
    again = graphs.batch_workload(candidates=12, degree=12, n_lo=512, n_hi=16384, base_nodes=4096, seed=3)
    assert all(np.array_equal(x.adj, y.adj) for x, y in zip(w, again))
