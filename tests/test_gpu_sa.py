"""Device annealing: every reported state is the exact evaluation of the
graph the device holds, and the graph stays simple and regular."""
import numpy as np
import pytest

import graphgolf_b200 as gg
import oracle
from graphgolf_b200 import graphs

pytestmark = pytest.mark.gpu


def _exact(g, edges):
    """(diameter, total) of the edges by the oracle (the CPU restatement of the
    reference's evaluation()); the GPU evaluator must agree."""
    adj = graphs.create_adj(g.nodes, g.degree, edges)
    h = graphs.Graph(g.nodes, g.degree, edges, adj)
    assert graphs.verify(h) == 0
    ok, diam, _, total = oracle.general(adj)
    r = gg.evaluate(adj)
    assert (r.diameter, r.total) == (diam, total)
    return diam, total


def _check(an, g, st):
    assert _exact(g, an.edges()) == (st.cur_diam, st.cur_total)
    assert _exact(g, an.edges(best=True)) == (st.best_diam, st.best_total)


@pytest.mark.parametrize("K,G,comp", [(1, 1, 0), (8, 8, 0), (16, 16, 8), (32, 256, 16)])
def test_hill_climbing_states_exact(gpu, K, G, comp):
    g = graphs.random_regular(512, 6, 11)
    with gg.Annealer(g, candidates=K, proposals=G, compose=comp, seed=3) as an:
        st0 = an.run(0)
        assert (st0.cur_diam, st0.cur_total) == _exact(g, g.edges)
        prev = st0.cur_total
        for _ in range(3):
            st = an.run(10)
            assert st.cur_total <= prev and st.cur_total == st.best_total
            prev = st.cur_total
            _check(an, g, st)
        assert st.step == 30 and st.evals >= 30 * K
        if comp:
            assert st.moved_swaps >= st.accepts
        assert st.cur_total < st0.cur_total


@pytest.mark.parametrize("n,d,K", [(300, 5, 16), (2048, 12, 64), (5000, 7, 32), (16384, 12, 64)])
def test_delta_evaluation_exact(gpu, n, d, K):
    """Candidates evaluated against the base equal their full evaluation,
    before and after the base is rebuilt by accepted moves."""
    g = graphs.random_regular(n, d, n + d)
    with gg.Annealer(g, candidates=K, compose=8, seed=6) as an:
        for rounds in range(3):
            c, m, u = an.check_delta()
            assert m == 0 and c + u == K and c >= K // 2
            an.run(3)
        st = an.run(0)
        assert st.delta
        _check(an, g, st)


def test_large_diameter_graph(gpu):
    """A random 3-regular graph of 20000 vertices (diameter above 15): the
    base keeps as many levels as the initial diameter, whatever the delta
    path serves agrees with the full evaluation, and the annealer (on the
    delta path or, where it would not serve, in full) accepts moves with
    exact states."""
    g = graphs.random_regular(20000, 3, 5)
    assert gg.evaluate(g.adj).diameter > 15
    with gg.Annealer(g, candidates=32, compose=8, seed=2) as an:
        c, m, u = an.check_delta()
        assert m == 0 and c + u == 32
        st = an.run(5)
        # a swap of a sparse graph of large diameter changes most distances: the
        # annealer measured that at creation and evaluates its candidates in full
        assert st.delta == (u * 4 <= 32)
        assert st.accepts > 0
        _check(an, g, st)


def _ladder(rungs):
    """A ladder of `rungs` rungs closed at each end by a K4 less one edge:
    3-regular and path-like (diameter about rungs + 3), its middle vertices of
    eccentricity about half of that."""
    e = []
    for i in range(rungs):
        e.append((i, rungs + i))
        if i + 1 < rungs:
            e += [(i, i + 1), (rungs + i, rungs + i + 1)]
    n = 2 * rungs
    for o, m in [(0, rungs), (rungs - 1, 2 * rungs - 1)]:
        p, q, r, s = n, n + 1, n + 2, n + 3
        e += [(p, r), (p, s), (q, r), (q, s), (r, s), (o, p), (m, q)]
        n += 4
    e = np.array(e, dtype=np.int32)
    return graphs.Graph(n, 3, e, graphs.create_adj(n, 3, e))


def _prism(k):
    """Two k-cycles joined by spokes: 3-regular, every eccentricity k/2 + 1."""
    e = [(i, (i + 1) % k) for i in range(k)] + [(k + i, k + (i + 1) % k) for i in range(k)] + \
        [(i, k + i) for i in range(k)]
    e = np.array(e, dtype=np.int32)
    return graphs.Graph(2 * k, 3, e, graphs.create_adj(2 * k, 3, e))


def test_levels_past_the_statistics(gpu):
    """The per-vertex statistics keep 32 levels.  A ladder of diameter about
    39: the base keeps every level, and candidates whose endpoints all lie
    within 31 of every vertex are served on levels past 32 and equal their
    full evaluation; the others are not served, never wrong.  A prism whose
    every eccentricity is 33: no candidate is served, so the annealer
    evaluates in full."""
    g = _ladder(36)
    assert 33 <= gg.evaluate(g.adj).diameter <= 45
    with gg.Annealer(g, candidates=128, compose=8, seed=4) as an:
        c, m, u = an.check_delta()
        assert m == 0 and c + u == 128 and c > 0
        _check(an, g, an.run(3))
    g = _prism(64)
    assert gg.evaluate(g.adj).diameter == 33
    with gg.Annealer(g, candidates=16, compose=4, seed=5) as an:
        c, m, u = an.check_delta()
        assert m == 0 and c == 0 and u == 16
        st = an.run(3)
        assert not st.delta
        _check(an, g, st)


def test_metropolis_states_exact(gpu):
    g = graphs.random_regular(400, 5, 4)
    with gg.Annealer(g, candidates=4, seed=9) as an:
        an.schedule(temp=200.0, cooling=0.98, hill_climbing=False)
        st = an.run(60)
        assert st.step == 60 and abs(st.temp - 200.0 * 0.98 ** 60) < 1e-9 * 200
        _check(an, g, st)
        assert st.best_total <= st.cur_total


def test_profile_matches_bfs(gpu):
    g = graphs.random_regular(300, 5, 2)
    with gg.Annealer(g, candidates=16, proposals=64, compose=4, seed=5) as an:
        assert np.array_equal(an.profile(), oracle.level_stats(g.adj))
        an.run(20)
        adj = graphs.create_adj(g.nodes, g.degree, an.edges())
        assert np.array_equal(an.profile(), oracle.level_stats(adj))


def test_target_stops_the_loop(gpu):
    g = graphs.random_regular(512, 6, 12)
    with gg.Annealer(g, candidates=16, compose=8, seed=2) as an:
        st0 = an.run(0)
        goal = st0.cur_total - 200
        an.target(st0.cur_diam, goal)
        st = st0
        for _ in range(50):
            st = an.run(8)
            if st.done:
                break
        assert st.done and st.cur_total <= goal
        again = an.run(8)
        assert (again.step, again.cur_total) == (st.step, st.cur_total)
        _check(an, g, again)


def test_large_learned_step(gpu):
    """The filter's full configuration: 4096 proposals, 64 evaluated."""
    g = graphs.random_regular(2048, 12, 7)
    with gg.Annealer(g, candidates=64, proposals=4096, compose=32, seed=4) as an:
        st = an.run(6)
        _check(an, g, st)
        assert st.evals == 6 * (64 + 4 + 1)   # candidates, predicted composites, exact composite


def test_bad_inputs(gpu):
    g = graphs.random_regular(64, 4, 1)
    bad = g.edges.copy()
    bad[0, 1] = bad[0, 0]                        # self-loop
    with pytest.raises(gg.EvaluationError):
        gg.Annealer(graphs.Graph(g.nodes, g.degree, bad, g.adj))
    with pytest.raises(gg.EvaluationError):
        gg.Annealer(g, candidates=0)
    with pytest.raises(gg.EvaluationError):
        gg.Annealer(g, candidates=16, proposals=100)   # not a multiple of 16
    with pytest.raises(gg.EvaluationError):
        gg.Annealer(g, candidates=10, proposals=64)    # filtered candidates: multiple of 16
    two = np.concatenate([g.edges, g.edges + 64])       # two components
    gd = graphs.Graph(128, 4, two.astype(np.int32), graphs.create_adj(128, 4, two))
    with pytest.raises(gg.EvaluationError):
        gg.Annealer(gd)


def test_filter_beats_random_selection(gpu):
    """What the trained network gains: after online training, the swaps it
    ranks highest improve the exact distance total far more often than the
    swaps drawn at random in the same steps (the last quarter of every
    step's evaluated candidates), and their exact changes are lower."""
    g = graphs.random_regular(2048, 12, 2)
    K = 64
    nt = K - K // 4
    with gg.Annealer(g, candidates=K, proposals=4096, compose=64, seed=1) as an:
        an.run(150)                                  # online training
        top, rnd = [], []
        for _ in range(60):
            an.run(1)
            p, lab = an.last_step()
            top.append(lab[:nt])
            rnd.append(lab[nt:])
        top, rnd = np.concatenate(top), np.concatenate(rnd)
        assert np.mean(top < 0) > 1.5 * np.mean(rnd < 0)
        assert top.mean() < rnd.mean()
        _check(an, g, an.run(0))


def _check_symmetric(an, g, st):
    """Both reported states are exact, and the edges the device holds are
    simple, regular and in the symmetric line order (line k*BL + i is line i
    shifted by k*B), so the graph really has the symmetry its group-weighted
    evaluation assumes: the oracle's full evaluation (every source) agrees."""
    B, n = g.nodes // g.groups, g.nodes
    for best, want in ((False, (st.cur_diam, st.cur_total)), (True, (st.best_diam, st.best_total))):
        e = an.edges(best=best)
        BL = e.shape[0] // g.groups
        for k in range(1, g.groups):
            assert np.array_equal(e[k * BL:(k + 1) * BL], (e[:BL] + k * B) % n)
        adj = graphs.create_adj(n, g.degree, e)
        assert graphs.verify(graphs.Graph(n, g.degree, e, adj)) == 0
        _, diam, _, total = oracle.general(adj, groups=g.groups)
        assert (diam, total) == want
        assert oracle.general(adj)[1::2] == (diam, total)


@pytest.mark.parametrize("n,d,grp,K,comp", [(2048, 8, 4, 1, 0), (2048, 8, 16, 16, 8), (1500, 6, 3, 8, 4),
                                            (4096, 12, 2, 32, 16)])
def test_symmetric_states_exact(gpu, n, d, grp, K, comp):
    """Orbit moves (2g-opt and 1g-opt) keep the graph symmetric; candidates are
    evaluated over n/groups sources, every state equals the oracle's."""
    g = graphs.symmetric_regular(n, d, grp, 30 + grp)
    with gg.Annealer(g, candidates=K, compose=comp, seed=9) as an:
        st0 = an.run(0)
        _, diam, _, total = oracle.general(g.adj, groups=grp)
        assert (st0.cur_diam, st0.cur_total) == (diam, total)
        prev = st0.cur_total
        for _ in range(3):
            st = an.run(15)
            assert st.cur_total <= prev
            prev = st.cur_total
            _check_symmetric(an, g, st)
        assert st.accepts > 0 and not st.delta
        assert st.cur_total < st0.cur_total


def test_symmetric_metropolis_states_exact(gpu):
    g = graphs.symmetric_regular(1024, 6, 8, 3)
    with gg.Annealer(g, candidates=4, seed=2) as an:
        an.schedule(50.0, 0.98, hill_climbing=False)
        for _ in range(3):
            st = an.run(20)
            _check_symmetric(an, g, st)


@pytest.mark.parametrize("K,G,comp", [(1, 1, 0), (32, 32, 8), (32, 256, 16)])
def test_grid_states_exact(gpu, K, G, comp):
    """Grid graphs: every move keeps both new edges within the length limit
    (grid/sa.c:137-221); every state equals the oracle's grid evaluation,
    plain, batched (delta path) and with the proposal filter."""
    w = h = 30
    g = graphs.grid_regular(w, h, 4, 3, 7)
    rh = graphs.rotate_hash(g.nodes, h, w, 1)
    with gg.Annealer(g, candidates=K, proposals=G, compose=comp, seed=5) as an:
        an.grid(h, 3)
        st0 = an.run(0)
        prev = st0.cur_total
        for _ in range(3):
            st = an.run(10)
            assert st.cur_total <= prev
            prev = st.cur_total
            for best, want in ((False, (st.cur_diam, st.cur_total)), (True, (st.best_diam, st.best_total))):
                e = an.edges(best=best)
                adj = graphs.create_adj(g.nodes, 4, e)
                assert graphs.verify(graphs.Graph(g.nodes, 4, e, adj, width=w, height=h), max_len=3) == 0
                ok, diam, _, total = oracle.grid(adj, rh)
                assert ok and (diam, total) == want
        assert st.cur_total < st0.cur_total


def test_orbit_and_grid_inputs_rejected(gpu):
    g = graphs.symmetric_regular(512, 6, 4, 1)
    bad = graphs.Graph(g.nodes, g.degree, g.edges[::-1].copy(), g.adj, groups=4)
    with pytest.raises(gg.EvaluationError):
        gg.Annealer(bad, candidates=4)
    with pytest.raises(ValueError):
        gg.Annealer(g, candidates=16, proposals=64)
    with gg.Annealer(g, candidates=4) as an:
        with pytest.raises(gg.EvaluationError):
            an.grid(16, 3)   # no length limits on symmetric graphs
    gr = graphs.grid_regular(20, 20, 4, 3, 2)
    with gg.Annealer(gr, candidates=4) as an:
        with pytest.raises(gg.EvaluationError):
            an.grid(20, 1)   # the current graph already has longer edges


@pytest.mark.parametrize("K,G,comp,metropolis", [(1, 1, 0, True), (16, 16, 8, False), (32, 256, 16, True)])
def test_checkpoint_resume_identical(gpu, K, G, comp, metropolis):
    """A run saved after 15 steps and resumed in a fresh annealer continues
    step for step: the same counters, temperature, current and best graphs as
    the run that was never interrupted (the step count keys the device's
    random stream; with a filter, the network's parameters and Adam state
    travel in the checkpoint too)."""
    g = graphs.random_regular(1024, 8, 5)

    def make(graph):
        an = gg.Annealer(graph, candidates=K, proposals=G, compose=comp, seed=9)
        if metropolis:
            an.schedule(temp=40.0, cooling=0.97, hill_climbing=False)
        return an

    with make(g) as a:
        a.run(15)
        ck = a.save()
        full = a.run(15)
        cur, best = a.edges(), a.edges(best=True)
    g2 = gg.checkpoint_graph(ck)
    assert g2.nodes == g.nodes and g2.degree == g.degree
    with make(g2) as b:
        b.restore(ck)
        resumed = b.run(15)
        assert resumed == full
        assert np.array_equal(b.edges(), cur) and np.array_equal(b.edges(best=True), best)
        _check(b, g, resumed)


def test_checkpoint_rejects_other_annealers(gpu):
    g = graphs.random_regular(512, 6, 2)
    with gg.Annealer(g, candidates=8, seed=1) as a:
        assert a.run(20).accepts > 0
        ck = a.save()
    with gg.Annealer(g, candidates=8, seed=1) as b:      # not the checkpoint's current graph
        with pytest.raises(gg.EvaluationError):
            b.restore(ck)
    with gg.Annealer(gg.checkpoint_graph(ck), candidates=16, seed=1) as c:   # another configuration
        with pytest.raises(gg.EvaluationError):
            c.restore(ck)
    bad = bytearray(ck)
    bad[0] ^= 0xFF
    with pytest.raises(gg.EvaluationError):
        gg.checkpoint_graph(bytes(bad))


def test_checkpoint_with_another_level_cap(gpu):
    """A checkpoint whose base kept more levels than the resuming annealer's
    first graph needs (its run started from a graph of larger diameter): the
    restore re-sizes the base to the saved cap and rebuilds it, and the
    resumed run's states are exact.  The cap is the header's 15th 32-bit
    field; raising it by one stands in for a run whose diameter has dropped."""
    import struct
    g = graphs.random_regular(1024, 8, 6)
    with gg.Annealer(g, candidates=16, compose=8, seed=4) as a:
        a.run(10)
        ck = bytearray(a.save())
    cap = struct.unpack_from("<i", ck, 56)[0]
    assert cap >= 2
    struct.pack_into("<i", ck, 56, cap + 1)
    with gg.Annealer(gg.checkpoint_graph(bytes(ck)), candidates=16, compose=8, seed=4) as b:
        b.restore(bytes(ck))
        st = b.run(10)
        assert st.step == 20
        _check(b, g, st)
        compared, bad, _ = b.check_delta()
        assert compared > 0 and bad == 0
