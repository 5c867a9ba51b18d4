"""The oracle itself: the C restatement (port) is pinned against the
reference's evaluator compiled from its own sources (oracle/_ref), against
the committed golden answers, against an independent queue BFS, and the
reference build is pinned against the reference's own golden log."""
import re
import subprocess

import numpy as np
import pytest

import oracle
from graphgolf_b200 import graphs
from _cases import aspl_of, build, case_id, golden_cases

SMALL = [c for c in golden_cases() if c["nodes"] <= 12000]
LARGE = [c for c in golden_cases() if c["nodes"] > 12000]


def _port(c, adj, rh):
    if c["kind"] == "grid":
        return oracle.grid(adj, rh, groups=c["groups"])
    n = adj.shape[0]
    return oracle.general(adj, based_nodes=(n - c["added_centers"]) // c["groups"], groups=c["groups"],
                          added_centers=c["added_centers"])


@pytest.mark.parametrize("c", SMALL, ids=case_id)
def test_port_matches_golden(c):
    adj, rh = build(c)
    ok, diam, aspl, total = _port(c, adj, rh)
    e = c["expected"]
    assert ok == e["connected"]
    assert diam == e["diameter"]
    if ok:
        assert aspl == aspl_of(c)          # bit-exact double
        assert total == e["total"]
    elif c["kind"] != "grid":
        assert aspl == aspl_of(c)          # DBL_MAX


@pytest.mark.slow
@pytest.mark.parametrize("c", LARGE, ids=case_id)
def test_port_matches_golden_large(c):
    test_port_matches_golden(c)


@pytest.mark.parametrize("algo", [1, 2])
@pytest.mark.parametrize("n,d,g,ac,seed", [(200, 5, 1, 0, 3), (4200, 6, 1, 0, 4), (600, 4, 4, 0, 5),
                                           (5000, 7, 2, 100, 6), (9000, 6, 1, 0, 8)])
def test_port_vs_reference_build(ref_oracle, algo, n, d, g, ac, seed):
    adj = graphs.random_regular(n, d, seed).adj
    bn = (n - ac) // g
    ok, diam, aspl, total = oracle.general(adj, based_nodes=bn, groups=g, added_centers=ac, algo=algo)
    assert (ok, diam, aspl) == oracle.ref_general(adj, based_nodes=bn, groups=g, added_centers=ac, algo=algo)


@pytest.mark.parametrize("procs", [2, 3, 5])
def test_partials_match_reference_ranks(ref_oracle, procs):
    """The MPI split (general/evaluation.c:166): rank r of `procs` through the
    reference build and through the port give the same partial sum/diameter,
    and the partials reduce to the one-rank answer."""
    n, d = 700, 6
    adj = graphs.random_regular(n, d, 11).adj
    full = oracle.general(adj)
    dmax, ssum = 1, 0
    for r in range(procs):
        dp, sp = oracle.general_partial(adj, r, procs)
        ok, diam, aspl = oracle.ref_general(adj, procs=procs, rank=r)
        assert diam == dp
        assert int(round(aspl * n * (n - 1))) - n * (n - 1) == sp
        dmax, ssum = max(dmax, dp), ssum + sp
    assert dmax == full[1]
    assert ssum + n * (n - 1) == full[3]


def test_bfs_oracle_agrees():
    for n, d, s in [(50, 3, 1), (300, 5, 2), (1024, 8, 1)]:
        adj = graphs.random_regular(n, d, s).adj
        ok, diam, aspl, total = oracle.general(adj)
        ecc, dsum = oracle.bfs_sums(adj)
        assert ok and ecc == diam and dsum == total


def test_bfs_oracle_grid_relabel():
    g = graphs.grid_regular(12, 12, 4, 3, 9)
    rh = graphs.rotate_hash(g.nodes, 12, 12, 4)
    ok, diam, aspl, total = oracle.grid(g.adj, rh, groups=4)
    ecc, dsum = oracle.bfs_sums(g.adj, n_sources=g.nodes // 4, relabel=rh)
    assert ok and dsum * 4 == total


def _ref_files(reference_tree, sub):
    return sorted((reference_tree / sub / "data").glob("*.edges"))


def test_port_vs_reference_on_its_data_files(reference_tree, ref_oracle):
    """Every general/data file that the reference reads with -M (symmetric
    ones with their -g), evaluated by the port and by the reference build."""
    checked = 0
    for f in _ref_files(reference_tree, "general"):
        m = re.search(r"g(\d+)", f.name)
        g = int(m.group(1)) if m else 1
        try:
            gr = graphs.read_general(str(f), groups=g)
        except ValueError:
            continue
        if gr.nodes > 6000 or gr.nodes % g or gr.degree * gr.nodes != 2 * gr.lines:
            continue
        ok, diam, aspl, total = oracle.general(gr.adj, groups=g)
        assert (ok, diam, aspl) == oracle.ref_general(gr.adj, groups=g), f.name
        checked += 1
    assert checked >= 50


def test_port_vs_reference_on_grid_files(reference_tree, ref_oracle):
    checked = 0
    for f in _ref_files(reference_tree, "grid"):
        gr = graphs.read_grid(str(f))
        ok, diam, aspl, total = oracle.grid(gr.adj, gr.rotate_hash)
        assert (ok, diam, aspl) == oracle.ref_grid(gr.adj, gr.rotate_hash), f.name
        checked += 1
    assert checked >= 10


def test_known_answers_from_reference_data(reference_tree, ref_oracle):
    """Values the reference programs print for their own data files at step 0
    (gg -f n256d4g64.edges -M -g 64; gg_grid -f w100h100d4.random.edges -R 200)."""
    g = graphs.read_general(str(reference_tree / "general/data/n256d4g64.edges"), groups=64)
    ok, diam, aspl, _ = oracle.general(g.adj, groups=64)
    assert (ok, diam, round(aspl, 6)) == (True, 6, 4.168627)
    w = graphs.read_grid(str(reference_tree / "grid/data/w100h100d4.random.edges"))
    ok, diam, aspl, _ = oracle.grid(w.adj, w.rotate_hash)
    assert (ok, diam, round(aspl, 6)) == (True, 11, 7.727035)


def test_reference_build_reproduces_its_golden_log(reference_tree, ref_oracle):
    """Pins oracle/_ref: the reference's own regression (general/Makefile:68-81)
    for the runs its golden log still matches (-v 16 -g 15, added centres)."""
    golden = (reference_tree / "general/data/result.txt").read_text().splitlines()
    finals = [l for l in golden if l.startswith("Diam. k =")]
    want = [l for l in finals if "2.883" in l or "2.88" in l]
    gg = oracle.REF_DIR / "gg"
    got = []
    for s in range(1, 11):
        out = subprocess.run([str(gg), "-f", str(reference_tree / "general/data/n114d29.random.edges"),
                              "-s", str(s), "-n", "100", "-v", "16", "-g", "15"], capture_output=True,
                             text=True, timeout=120).stdout
        got.append([l for l in out.splitlines() if l.startswith("Diam. k =")][-1])
    # the ten -v 16 -g 15 finals are the last line of each seed's block in result.txt
    blocks = [finals[i] for i in range(7, len(finals), 8)]
    assert got == blocks[:10]


@pytest.mark.parametrize("n,d,drop,g,ac,algo", [(300, 6, 150, 1, 0, 1), (512, 8, 300, 4, 0, 2), (610, 5, 100, 2, 10, 1),
                                                (1000, 12, 2000, 1, 40, 1)])
def test_nonregular_port_vs_reference_build(n, d, drop, g, ac, algo):
    """The non-regular general variant (per-row degrees in the based phase,
    whole padded rows in the added-centre phase), port vs the reference build."""
    if not oracle.have_ref_nr():
        pytest.skip("oracle/_ref non-regular builds absent")
    gr = graphs.random_regular(n, d, n + drop)
    _, adj, deg = graphs.nonregular(gr, drop, 7)
    bn = (n - ac) // g
    got = oracle.general_nr(adj, deg, based_nodes=bn, groups=g, added_centers=ac, algo=algo)
    assert got[:3] == oracle.ref_general_nr(adj, deg, based_nodes=bn, groups=g, added_centers=ac, algo=algo)


@pytest.mark.parametrize("w,h,d,drop,g", [(16, 16, 6, 100, 1), (20, 20, 4, 60, 2), (18, 18, 6, 120, 4)])
def test_nonregular_grid_port_vs_reference_build(w, h, d, drop, g):
    if not oracle.have_ref_nr():
        pytest.skip("oracle/_ref non-regular builds absent")
    gr = graphs.grid_regular(w, h, d, 3, w + drop)
    _, adj, deg = graphs.nonregular(gr, drop, 3)
    rh = graphs.rotate_hash(gr.nodes, h, w, g)
    got = oracle.grid_nr(adj, deg, rh, groups=g)
    assert got[:3] == oracle.ref_grid_nr(adj, deg, rh, groups=g)
