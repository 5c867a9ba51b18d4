"""The multi-rank path: two gloo ranks each take a strided share of the source
chunks and join the partial results with the all-reduces of
graphgolf_b200.distributed.  On the CPU the per-rank partial is the oracle's
(the reference's MPI split restated), standing in for the GPU partial, so
what is under test is the host-side decomposition and reduction; with a GPU
the same run uses the CUDA partials.  Either way the result must be the
one-rank answer exactly.  Also checks that a rank that never joins makes the
others fail with an error instead of hanging."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from graphgolf_b200 import graphs


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _oracle_partial(adj, rank, procs, based_nodes=None, groups=1, added_centers=0):
    import oracle
    from graphgolf_b200._native import ggb_partial
    diam, s = oracle.general_partial(adj, rank, procs, based_nodes=based_nodes, groups=groups,
                                     added_centers=added_centers)
    return ggb_partial(diam, 1 if diam > adj.shape[0] else 0, s, 0, 0, 0, 0)


def _gpu_partial_in_turn(adj, rank, procs, **kw):
    """The GPU partial of this rank (ggb_eval_general_partial on cuda:0).
    The ranks share one GPU here, so they take turns, each finishing its
    evaluation before the next starts; no kernel ever waits on another
    rank's."""
    import torch.distributed as dist
    from graphgolf_b200.evaluator import evaluate_partial
    p = None
    for r in range(procs):
        if r == rank:
            p = evaluate_partial(adj, rank, procs, **kw)
        dist.barrier()
    return p


def _worker(rank, world, port, cases, out, use_gpu=False):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from datetime import timedelta
    from graphgolf_b200.distributed import evaluate_sharded
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    res = []
    for adj, g, ac in cases:
        n = adj.shape[0]
        r = evaluate_sharded(adj, based_nodes=(n - ac) // g, groups=g, added_centers=ac,
                             partial_fn=_gpu_partial_in_turn if use_gpu else _oracle_partial)
        res.append((r.connected, r.diameter, r.aspl, r.total))
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()


def _cases():
    return [(graphs.random_regular(700, 6, 1).adj, 1, 0),
            (graphs.symmetric_regular(1024, 8, 4, 2).adj, 4, 0),
            (graphs.random_regular(610, 5, 3).adj, 2, 10)]


def test_two_gloo_ranks_match_one_rank():
    _run_two_ranks(use_gpu=False)


@pytest.mark.gpu
def test_two_gloo_ranks_with_gpu_partials_match_one_rank(gpu):
    """The same decomposition with each rank's partial computed by the CUDA
    path (ggb_eval_general_partial) instead of the oracle's."""
    _run_two_ranks(use_gpu=True)


def _run_two_ranks(use_gpu):
    import oracle
    cases = _cases()
    want = []
    for adj, g, ac in cases:
        n = adj.shape[0]
        want.append(oracle.general(adj, based_nodes=(n - ac) // g, groups=g, added_centers=ac))
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, cases, out, use_gpu)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        assert out[r] == want


def _lonely(rank, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    try:
        store = dist.TCPStore("127.0.0.1", port, 2, rank == 0, timeout=timedelta(seconds=3))
        dist.init_process_group("gloo", store=store, rank=rank, world_size=2, timeout=timedelta(seconds=3))
        t = torch.zeros(1)
        dist.all_reduce(t)
        out[rank] = "joined"
    except Exception as e:  # the peer never arrives: a bounded failure, not a hang
        out[rank] = type(e).__name__


def test_missing_rank_fails_instead_of_hanging():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    p = ctx.Process(target=_lonely, args=(0, _free_port(), out))
    p.start()
    p.join(timeout=60)
    assert p.exitcode == 0
    assert out[0] != "joined"
