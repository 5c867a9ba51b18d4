"""Parity of the CUDA path (through the C ABI) with the oracle.

Bar: bit-exact.  The diameter, the connectivity flag and the integer distance
total must be identical, and ASPL must be the identical double (it is the
same expression of the same integer)."""
import numpy as np
import pytest

import graphgolf_b200 as gg
import oracle
from graphgolf_b200 import graphs
from _cases import aspl_of, build, case_id, golden_cases, union_graph

pytestmark = pytest.mark.gpu


def _gpu(c, adj, rh):
    n = adj.shape[0]
    if c["kind"] == "grid":
        return gg.evaluate_grid(adj, rh, groups=c["groups"])
    return gg.evaluate(adj, based_nodes=(n - c["added_centers"]) // c["groups"], groups=c["groups"],
                       added_centers=c["added_centers"])


@pytest.mark.parametrize("c", golden_cases(), ids=case_id)
def test_golden(gpu, c):
    """Every known answer of the reference build (tests/golden)."""
    adj, rh = build(c)
    r = _gpu(c, adj, rh)
    e = c["expected"]
    assert r.connected == e["connected"]
    assert r.diameter == e["diameter"]
    if r.connected:
        assert r.total == e["total"]
        assert r.aspl == aspl_of(c)
    elif c["kind"] != "grid":
        assert r.aspl == aspl_of(c)


@pytest.mark.parametrize("n,d,seed", [(4, 3, 1), (6, 3, 2), (8, 7, 3), (33, 4, 4), (65, 2, 5), (127, 4, 6),
                                      (128, 5, 7), (129, 6, 8), (300, 9, 9), (1025, 6, 10), (3000, 33, 11),
                                      (8192, 10, 12), (10001, 4, 13)])
def test_random_vs_oracle(gpu, n, d, seed):
    adj = graphs.random_regular(n, d, seed).adj
    ok, diam, aspl, total = oracle.general(adj)
    r = gg.evaluate(adj)
    assert (r.connected, r.diameter, r.aspl, r.total) == (ok, diam, aspl, total)


@pytest.mark.parametrize("bits", [64, 128, 256, 512, 1024, 2048, 4096, 8192])
def test_window_width_sweep(gpu, bits):
    """Results never depend on the window width or the grid size."""
    adj = graphs.random_regular(3000, 7, 21).adj
    want = oracle.general(adj)
    try:
        for ctas in (0, 1, 3):
            gg.set_tuning(bits, ctas)
            r = gg.evaluate(adj)
            assert (r.connected, r.diameter, r.aspl, r.total) == want
            assert r.window_bits == bits
    finally:
        gg.set_tuning(0, 0)


@pytest.mark.parametrize("g", [2, 4, 8, 16, 32])
def test_symmetric_groups(gpu, g):
    s = graphs.symmetric_regular(2048, 8, g, 40 + g)
    want = oracle.general(s.adj, groups=g)
    r = gg.evaluate(s.adj, groups=g)
    assert (r.connected, r.diameter, r.aspl, r.total) == want


@pytest.mark.parametrize("n,d,g,ac", [(1040, 8, 16, 16), (300, 5, 3, 30), (5000, 8, 1, 700), (2050, 6, 8, 2)])
def test_added_centres(gpu, n, d, g, ac):
    adj = graphs.random_regular(n, d, n + ac).adj
    bn = (n - ac) // g
    want = oracle.general(adj, based_nodes=bn, groups=g, added_centers=ac)
    r = gg.evaluate(adj, based_nodes=bn, groups=g, added_centers=ac)
    assert (r.connected, r.diameter, r.aspl, r.total) == want


@pytest.mark.parametrize("n,d", [(8, 3), (100, 4), (1000, 3), (5000, 6)])
def test_disconnected(gpu, n, d):
    adj = union_graph(n, d, 77)
    r = gg.evaluate(adj)
    assert (r.connected, r.diameter, r.aspl) == oracle.general(adj)[:3]
    assert r.diameter == 2**31 - 1 and r.aspl == np.finfo(np.float64).max
    # grid convention: diameter nodes+1, ASPL untouched
    ok, diam, aspl = gg.grid_evaluation(2 * n, d, 1, adj, 2 * n, 1, 1, False, np.arange(2 * n), aspl_in=3.5)
    assert (ok, diam, aspl) == (False, 2 * n + 1, 3.5)
    assert oracle.grid(adj, np.arange(2 * n))[:2] == (False, 2 * n + 1)


def test_isolated_and_tiny(gpu):
    # a single edge: N=2, d=1
    adj = np.array([[1], [0]], dtype=np.int32)
    assert gg.evaluation(2, 2, 1, 1, 1, adj) == oracle.general(adj)[:3]
    # N=1, d=0: the reference reports it disconnected (diam 1 is not < 1)
    adj = np.zeros((1, 0), dtype=np.int32)
    assert gg.evaluation(1, 1, 1, 0, 0, adj) == oracle.general(adj)[:3]
    # complete graph K5
    adj = np.array([[j for j in range(5) if j != i] for i in range(5)], dtype=np.int32)
    assert gg.evaluation(5, 5, 1, 10, 4, adj) == oracle.general(adj)[:3]


@pytest.mark.parametrize("w,h,d,r,g", [(10, 10, 4, 3, 1), (20, 20, 6, 3, 2), (32, 32, 4, 3, 4), (50, 40, 4, 2, 1)])
def test_grid_vs_oracle(gpu, w, h, d, r, g):
    gr = graphs.grid_regular(w, h, d, r, w + h + g)
    rh = graphs.rotate_hash(gr.nodes, h, w, g)
    want = oracle.grid(gr.adj, rh, groups=g)
    res = gg.evaluate_grid(gr.adj, rh, groups=g)
    assert (res.connected, res.diameter, res.total) == (want[0], want[1], want[3])
    assert res.aspl == want[2]


def test_repeated_calls_identical(gpu):
    """Back-to-back evaluations of different sizes reuse the grow-only buffers."""
    a = graphs.random_regular(5000, 8, 1).adj
    b = graphs.random_regular(300, 5, 2).adj
    ra, rb = oracle.general(a), oracle.general(b)
    for _ in range(3):
        for adj, want in ((a, ra), (b, rb)):
            r = gg.evaluate(adj)
            assert (r.connected, r.diameter, r.aspl, r.total) == want


def test_large_properties(gpu):
    """The headline-size graph (N=65536, d=16): the GPU total equals the golden, and the symmetric
    g=16 variant runs 1/16 of the sources yet gives the same-size total."""
    for c in golden_cases():
        if c["nodes"] == 65536:
            adj, rh = build(c)
            r = _gpu(c, adj, rh)
            assert (r.diameter, r.total) == (c["expected"]["diameter"], c["expected"]["total"])
            assert r.windows == -(-65536 // c["groups"] // r.window_bits)


def _headline_cases():
    return [c for c in golden_cases() if c["nodes"] == 65536]


@pytest.mark.parametrize("bits", [64, 128, 256, 512, 0])
@pytest.mark.parametrize("c", _headline_cases(), ids=case_id)
def test_headline_graph_at_every_width(gpu, c, bits):
    """The single-large-evaluation configuration at its size: the seeded
    16-regular graph with N=65536 (g=1, all 65536 sources) and its rotationally
    symmetric variant (g=16, 4096 sources), at source-window widths of 64,
    128, 256 and 512 bits and the automatic width, against the reference
    build's own answer (tests/golden)."""
    adj, rh = build(c)
    try:
        gg.set_tuning(bits, 0)
        r = _gpu(c, adj, rh)
    finally:
        gg.set_tuning(0, 0)
    e = c["expected"]
    assert (r.connected, r.diameter, r.total) == (e["connected"], e["diameter"], e["total"])
    assert r.aspl == aspl_of(c)
    if bits:
        assert r.window_bits == bits
    assert r.windows == -(-65536 // c["groups"] // r.window_bits)


@pytest.mark.parametrize("ball", [0, 1])
@pytest.mark.parametrize("bits", [64, 128, 1024, 4096])
@pytest.mark.parametrize("n,d,g,ac", [(3000, 7, 1, 0), (3000, 8, 1, 0), (2400, 12, 4, 0), (1040, 8, 16, 16),
                                      (5000, 5, 1, 100), (700, 32, 1, 0)])
def test_seeding_paths(gpu, ball, bits, n, d, g, ac):
    """Both ways of starting a window -- the per-window two-hop seeding and
    the ball pre-pass -- with scalar (odd degree) and vector adjacency loads,
    over one and many windows, give the oracle's answer."""
    adj = graphs.random_regular(n, d, n + d + g).adj
    bn = (n - ac) // g
    want = oracle.general(adj, based_nodes=bn, groups=g, added_centers=ac)
    try:
        gg.set_ball(ball)
        gg.set_tuning(bits, 0)
        r = gg.evaluate(adj, based_nodes=bn, groups=g, added_centers=ac)
    finally:
        gg.set_ball(-1)
        gg.set_tuning(0, 0)
    assert (r.connected, r.diameter, r.aspl, r.total) == want


@pytest.mark.parametrize("ball", [0, 1])
def test_seeding_paths_grid_and_disconnected(gpu, ball):
    try:
        gg.set_ball(ball)
        gg.set_tuning(256, 0)
        gr = graphs.grid_regular(30, 30, 4, 3, 5)
        rh = graphs.rotate_hash(gr.nodes, 30, 30, 2)
        want = oracle.grid(gr.adj, rh, groups=2)
        res = gg.evaluate_grid(gr.adj, rh, groups=2)
        assert (res.connected, res.diameter, res.aspl, res.total) == want
        adj = union_graph(900, 6, 5)
        r = gg.evaluate(adj)
        assert (r.connected, r.diameter, r.aspl) == oracle.general(adj)[:3]
    finally:
        gg.set_ball(-1)
        gg.set_tuning(0, 0)
