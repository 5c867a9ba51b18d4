"""Batched evaluation: many graphs of uneven sizes in one launch.

Bar: every graph's result is bit-identical to the oracle's (and so to the
single-graph evaluator's) -- for every plan (window width x CTAs per team)."""
import numpy as np
import pytest

import graphgolf_b200 as gg
import oracle
from graphgolf_b200 import graphs
from _cases import union_graph

pytestmark = pytest.mark.gpu


def _mixed():
    """Uneven sizes, odd and even degrees, symmetric graphs and a
    disconnected one."""
    out = []   # (adj, groups)
    for n, d, s in [(4, 3, 1), (33, 4, 2), (129, 6, 3), (700, 5, 4), (1025, 12, 5), (3000, 7, 6), (5000, 12, 7)]:
        out.append((graphs.random_regular(n, d, s).adj, 1))
    for n, d, g in [(2048, 8, 16), (600, 6, 3)]:
        out.append((graphs.symmetric_regular(n, d, g, n + g).adj, g))
    out.append((union_graph(500, 4, 9), 1))
    out.append((np.array([[1], [0]], dtype=np.int32), 1))
    return out


def _want(adj, g):
    """The oracle's answer (the CPU restatement of the reference's evaluation())."""
    return oracle.general(adj, groups=g)


def _got(r):
    return (r.connected, r.diameter, r.aspl, r.total)


@pytest.fixture(scope="module")
def mixed():
    m = _mixed()
    return m, [_want(a, g) for a, g in m]


def test_mixed_matches_oracle(gpu, mixed):
    """The single-graph evaluator agrees with the oracle on every graph of the mix."""
    m, want = mixed
    for (adj, g), w in zip(m, want):
        r = gg.evaluate(adj, groups=g)
        assert (r.connected, r.diameter, r.aspl, r.total) == w


@pytest.mark.parametrize("bits", [128, 512, 4096])
@pytest.mark.parametrize("team", [1, 2, 5, 148])
def test_every_plan_identical(gpu, mixed, bits, team):
    m, want = mixed
    with gg.Batch([a.shape[0] for a, _ in m], [a.shape[1] for a, _ in m], [g for _, g in m]) as b:
        b.set_plan(bits, team)
        wb, tc, teams = b.plan
        assert wb == bits and tc == min(team, tc) and teams >= 1
        res = b.evaluate([a for a, _ in m])
        assert [_got(r) for r in res] == want
        assert all(r.window_bits == bits for r in res)


def test_graph_replay_tracks_contents(gpu):
    """The captured launch is replayed; results follow the uploaded arrays."""
    sizes = [800, 1500, 3000]
    a = [graphs.random_regular(n, 6, n).adj for n in sizes]
    c = [graphs.swap_2opt(graphs.random_regular(n, 6, n), 7).adj for n in sizes]
    with gg.Batch(sizes, 6) as b:
        for _ in range(2):
            assert [_got(r) for r in b.evaluate(a)] == [_want(x, 1) for x in a]
            assert [_got(r) for r in b.evaluate(c)] == [_want(x, 1) for x in c]


def test_autotune_keeps_results(gpu, mixed):
    m, want = mixed
    with gg.Batch([a.shape[0] for a, _ in m], [a.shape[1] for a, _ in m], [g for _, g in m]) as b:
        b.upload([a for a, _ in m])
        bits, team, ms = b.autotune(iters=1)
        assert bits % 128 == 0 and team >= 1 and ms > 0
        assert b.plan[:2] == (bits, team)
        b.launch()
        assert [_got(r) for r in b.collect()] == want
        assert b.kernel_ms() > 0


def test_device_stream_path(gpu):
    import torch
    sizes = [1000, 2000]
    a = [graphs.random_regular(n, 8, n + 3).adj for n in sizes]
    s = torch.cuda.Stream()
    with gg.Batch(sizes, 8) as b:
        b.upload(a, stream=s.cuda_stream)
        b.launch(stream=s.cuda_stream)
        assert [_got(r) for r in b.collect(stream=s.cuda_stream)] == [_want(x, 1) for x in a]
        # adjacency written in place on the device, through a torch view
        assert b.adj_ptr(0) % 16 == 0
        c = graphs.swap_2opt(graphs.random_regular(1000, 8, 1003), 11).adj
        v = b.adj_view(0)
        assert tuple(v.shape) == (1000, 8) and v.data_ptr() == b.adj_ptr(0)
        v.copy_(torch.from_numpy(c))
        torch.cuda.synchronize()
        b.launch()
        res = b.collect()
        assert _got(res[0]) == _want(c, 1)
        assert _got(res[1]) == _want(a[1], 1)


def test_bad_entry_reported_and_batch_reusable(gpu):
    sizes = [300, 400, 500]
    a = [graphs.random_regular(n, 4, n).adj for n in sizes]
    bad = [x.copy() for x in a]
    with gg.Batch(sizes, 4) as b:
        # 400 == nodes of graph 1 travels as a 16-bit id; 1 << 20 and -1 make
        # the upload fall back to plain ints.  All are caught on the device.
        for v in (400, 1 << 20, -1):
            bad[1][17, 2] = v
            with pytest.raises(gg.EvaluationError) as ei:
                b.evaluate(bad)
            assert ei.value.code == -3 and "graph 1" in str(ei.value), v
            assert [_got(r) for r in b.evaluate(a)] == [_want(x, 1) for x in a]


def test_bad_sizes_rejected(gpu):
    with pytest.raises(gg.EvaluationError):
        gg.Batch([10, 0], 3)
    with pytest.raises(gg.EvaluationError):
        gg.Batch([10, 12], 3, [3, 4])   # 10 is not a multiple of 3
    with gg.Batch([10], 3) as b:
        with pytest.raises(gg.EvaluationError):
            b.set_plan(192, 1)          # not 128 * 2^k
        with pytest.raises(gg.EvaluationError):
            b.evaluate([np.zeros((10, 2), dtype=np.int32)])


def test_uneven_workload_full_size(gpu):
    """The mixed workload at full size: a 4096-vertex 12-regular base graph
    and 256 single-swap candidates of 12-regular graphs with 512..16384
    vertices, each bit-identical to the single-graph evaluator."""
    w = graphs.batch_workload()
    with gg.Batch([x.nodes for x in w], 12) as b:
        res = b.evaluate([x.adj for x in w])
        for x, r in zip(w, res):
            assert _got(r) == _want(x.adj, 1)
    for x, r in list(zip(w, res))[:4]:
        if x.nodes <= 2048:
            assert _got(r) == oracle.general(x.adj)
