"""The drop-in's MPI split (libgg_general built with -DGGB_WITH_MPI): with
procs > 1 every rank evaluates its strided share of the source windows and
the ranks join diameter and distance sum with MPI_Allreduce, as the
reference's evaluation() does (general/evaluation.c:166,247-248).  Two
processes run the test driver (an MPI host in the reference's shape) with a
file-based two-rank MPI stand-in (tests/mpi_two_rank/mpi.h); both must print
the one-rank answer of the oracle.  On the CPU the per-rank partial comes from
a stand-in core library built on the oracle; with a GPU the real core
library runs it."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from graphgolf_b200 import graphs

ROOT = Path(__file__).resolve().parent.parent
STUB = ROOT / "tests" / "mpi_two_rank"
LIB = ROOT / "graphgolf_b200" / "_lib"
CC = ["gcc", "-std=gnu11", "-O2", "-fPIC", "-Wall", "-Wno-unused-parameter"]


def _build(tmp: Path, core: str) -> Path:
    """Builds the MPI shim and the driver against `core` ("fake" or "real")."""
    if core == "fake":
        subprocess.run(CC + ["-shared", "-o", str(tmp / "libgraphgolf_b200.so"), str(STUB / "fake_core.c"),
                             f"-L{oracle.HERE}", "-loracle", f"-Wl,-rpath,{oracle.HERE}"], check=True)
        core_dir = tmp
    else:
        core_dir = LIB
    subprocess.run(CC + ["-DGGB_WITH_MPI", f"-I{STUB}", "-shared", "-o", str(tmp / "libgg_general.so"),
                         str(ROOT / "graphgolf_b200" / "csrc" / "dropin_general.c"), f"-L{core_dir}",
                         "-lgraphgolf_b200", f"-Wl,-rpath,{core_dir}"], check=True)
    drv = tmp / "driver"
    subprocess.run(CC + [f"-I{STUB}", "-o", str(drv), str(STUB / "driver.c"), f"-L{tmp}", "-lgg_general",
                         f"-Wl,-rpath,{tmp}"], check=True)
    return drv


def _cases():
    return [(graphs.random_regular(700, 6, 1).adj, 1, 0),
            (graphs.symmetric_regular(1024, 8, 4, 2).adj, 4, 0),
            (graphs.random_regular(610, 5, 3).adj, 2, 10),
            (np.concatenate([graphs.random_regular(100, 4, 5).adj,
                             graphs.random_regular(100, 4, 6).adj + 100]).astype(np.int32), 1, 0)]


def _run_world(drv: Path, tmp: Path, adj, g, ac, size=2):
    n, d = adj.shape
    f = tmp / "adj.bin"
    np.ascontiguousarray(adj, dtype=np.int32).tofile(f)
    outs = []
    for trial in range(1):
        ex = tmp / f"x{trial}_{n}_{g}_{ac}"
        ex.mkdir()
        procs = []
        for r in range(size):
            env = dict(os.environ, GGB_TEST_RANK=str(r), GGB_TEST_SIZE=str(size), GGB_TEST_DIR=str(ex), OMP_NUM_THREADS="1")
            procs.append(subprocess.Popen([str(drv), str(f), str(n), str((n - ac) // g), str(g), str(d), str(ac)],
                                          stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env))
        for p in procs:
            o, e = p.communicate(timeout=300)
            assert p.returncode == 0, o + e
            outs.append(o.split())
    return outs


def _want(adj, g, ac):
    n = adj.shape[0]
    ok, diam, aspl, _ = oracle.general(adj, based_nodes=(n - ac) // g, groups=g, added_centers=ac)
    return [str(int(ok)), str(diam), float(aspl).hex()]


def test_mpi_split_with_stand_in_core(tmp_path):
    drv = _build(tmp_path, "fake")
    for adj, g, ac in _cases():
        outs = _run_world(drv, tmp_path, adj, g, ac)
        want = _want(adj, g, ac)
        for o in outs:
            assert [o[0], o[1], float.fromhex(o[2]).hex()] == want


@pytest.mark.gpu
def test_mpi_split_on_the_gpu(gpu, tmp_path):
    """Two ranks on one GPU, each running its share with the CUDA path; no
    kernel of one rank waits on the other's (they meet only on the host)."""
    drv = _build(tmp_path, "real")
    for adj, g, ac in _cases()[:3]:
        outs = _run_world(drv, tmp_path, adj, g, ac)
        want = _want(adj, g, ac)
        for o in outs:
            assert [o[0], o[1], float.fromhex(o[2]).hex()] == want
