"""The multi-rank decomposition on the GPU: ggb_eval_general_partial for rank
r of P runs source windows r, r+P, ... (the reference's MPI split,
general/evaluation.c:166; the added-centre windows start at
(r - based_nodes % P) mod P, :209-212) and must return exactly the oracle's
partial of the same rank and window width, for every rank.  The partials
joined as the reference's MPI_Allreduce joins them (MAX diameter, SUM sum,
:247-248) must give the one-rank answer."""
import pytest

import graphgolf_b200 as gg
import oracle
from graphgolf_b200 import graphs
from _cases import union_graph

pytestmark = pytest.mark.gpu


def _cases():
    return [
        ("random-g1", graphs.random_regular(3000, 8, 5).adj, 1, 0),
        ("symmetric-g16", graphs.symmetric_regular(4096, 12, 16, 8).adj, 16, 0),
        ("added-centres", graphs.random_regular(2050, 6, 9).adj, 8, 2),
        ("added-centres-g1", graphs.random_regular(5000, 8, 3).adj, 1, 700),
    ]


@pytest.mark.parametrize("bits", [64, 128, 512])
@pytest.mark.parametrize("procs", [2, 3, 8])
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_partial_of_every_rank_matches_oracle(gpu, case, procs, bits):
    _, adj, g, ac = case
    n = adj.shape[0]
    bn = (n - ac) // g
    diam, total, disc = 1, 0, 0
    try:
        gg.set_tuning(bits, 0)
        for r in range(procs):
            p = gg.evaluate_partial(adj, r, procs, based_nodes=bn, groups=g, added_centers=ac)
            assert p.window_bits == bits
            want = oracle.general_partial(adj, r, procs, based_nodes=bn, groups=g, added_centers=ac,
                                          window_bits=bits)
            assert (p.diam, p.sum) == want, f"rank {r} of {procs}"
            diam, total, disc = max(diam, p.diam), total + p.sum, max(disc, p.disconnected)
    finally:
        gg.set_tuning(0, 0)
    res = gg.finish_general(n, diam, disc, total)
    want = oracle.general(adj, based_nodes=bn, groups=g, added_centers=ac)
    assert (res.connected, res.diameter, res.aspl, res.total) == want


def test_partials_of_a_disconnected_graph(gpu):
    """Some rank finds the unreachable pair; the joined result is the
    reference's disconnected convention."""
    adj = union_graph(900, 6, 4)
    n = adj.shape[0]
    diam, disc, total = 1, 0, 0
    for r in range(3):
        p = gg.evaluate_partial(adj, r, 3)
        diam, disc, total = max(diam, p.diam), max(disc, p.disconnected), total + p.sum
    res = gg.finish_general(n, diam, disc, total)
    assert (res.connected, res.diameter, res.aspl) == oracle.general(adj)[:3]
