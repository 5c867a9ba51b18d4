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


def test_pure_python_generators_match_the_c_generators():
    """oracle.graphgen (used by bench.py's reference arm, which loads none of
    the package's libraries) draws the identical graphs."""
    from oracle import graphgen
    for n, d, s in [(500, 6, 3), (66, 5, 5), (1024, 8, 1), (3000, 7, 21)]:
        g = graphs.random_regular(n, d, s)
        e = graphgen.random_regular_edges(n, d, s)
        assert np.array_equal(e, g.edges)
        assert np.array_equal(graphgen.create_adj(n, d, e), g.adj)
    for n, d, gr, s in [(256, 6, 4, 2), (2048, 8, 16, 3)]:
        assert np.array_equal(graphgen.symmetric_regular_edges(n, d, gr, s), graphs.symmetric_regular(n, d, gr, s).edges)


def test_pure_python_generator_reproduces_the_headline_graphs():
    """The bench graphs (N=65536, d=16, g=1 and g=16) by their golden adjacency hashes."""
    import json
    import sys
    from pathlib import Path
    from oracle import graphgen
    gold = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(gold))
    from make_golden import adj_hash
    for c in json.loads((gold / "apsp_golden.json").read_text())["cases"]:
        if c["nodes"] != 65536:
            continue
        p = c["params"]
        if c["groups"] == 1:
            e = graphgen.random_regular_edges(p["n"], p["d"], c["seed"])
        else:
            e = graphgen.symmetric_regular_edges(p["n"], p["d"], c["groups"], c["seed"])
        assert adj_hash(graphgen.create_adj(p["n"], p["d"], e)) == c["adj_sha"]


def test_grid_trajectory_fixture_matches_the_generator(tmp_path):
    """The committed 100 000-step grid trajectory was recorded on the input
    the seeded lattice generator gives today, and holds one progress row per
    1 000 steps plus the final result lines."""
    import hashlib
    import json
    import sys
    from pathlib import Path
    gold = Path(__file__).resolve().parent / "golden"
    want = json.loads((gold / "grid_trajectory_w100h100d4r3.json").read_text())
    sys.path.insert(0, str(gold))
    from make_grid_trajectory import CONFIG, write_input
    assert want["config"] == CONFIG
    f = tmp_path / "in.edges"
    write_input(str(f))
    assert hashlib.sha256(f.read_bytes()).hexdigest() == want["input_sha256"]
    rows = [l for l in want["lines"] if l.split() and l.split()[0].isdigit()]
    assert [int(r.split()[0]) for r in rows] == list(range(0, CONFIG["steps"], 1000))
    assert any(l.startswith("Diam. k") for l in want["lines"])
    assert any(l.startswith("Accept rate") for l in want["lines"])
