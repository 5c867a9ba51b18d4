"""Host C code under AddressSanitizer and UndefinedBehaviorSanitizer (CPU).

The package's host library (graph_host.c: generators, edge files, adjacency,
checks), the oracle's C restatement, and the general drop-in shim (driven by
the test MPI host with a stand-in core library) are built with
-fsanitize=address,undefined and run on small graphs; any out-of-bounds
access, leak or undefined behaviour fails the run."""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from graphgolf_b200 import graphs

ROOT = Path(__file__).resolve().parent.parent
SAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=undefined", "-fno-omit-frame-pointer", "-g", "-O1"]
ENV = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0:halt_on_error=1",
           UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1", OMP_NUM_THREADS="2")

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is needed")


def _gcc(args):
    p = subprocess.run(["gcc", "-std=gnu11", *SAN, *args], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-3000:]


def test_host_and_oracle_under_sanitizers(tmp_path):
    exe = tmp_path / "harness"
    _gcc(["-fopenmp", "-o", str(exe), str(ROOT / "tests" / "sanitize" / "harness.c"),
          str(ROOT / "graphgolf_b200" / "csrc" / "host" / "graph_host.c"), str(ROOT / "oracle" / "apsp_oracle.c")])
    p = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, env=ENV, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    assert "ok" in p.stdout


def test_general_shim_under_sanitizers(tmp_path):
    """The general shim with its MPI split, one and two ranks."""
    stub = ROOT / "tests" / "mpi_two_rank"
    exe = tmp_path / "shim"
    _gcc(["-fopenmp", "-DGGB_WITH_MPI", f"-I{stub}", "-o", str(exe), str(stub / "driver.c"),
          str(ROOT / "graphgolf_b200" / "csrc" / "dropin_general.c"), str(stub / "fake_core.c"),
          str(ROOT / "oracle" / "apsp_oracle.c")])
    adj = graphs.random_regular(300, 5, 8).adj
    f = tmp_path / "adj.bin"
    np.ascontiguousarray(adj).tofile(f)
    ok, diam, aspl, _ = oracle.general(adj)
    for size in (1, 2):
        ex = tmp_path / f"x{size}"
        ex.mkdir()
        procs = [subprocess.Popen([str(exe), str(f), "300", "300", "1", "5", "0"], stdout=subprocess.PIPE,
                                  stderr=subprocess.PIPE, text=True,
                                  env=dict(ENV, GGB_TEST_RANK=str(r), GGB_TEST_SIZE=str(size), GGB_TEST_DIR=str(ex)))
                 for r in range(size)]
        for p in procs:
            o, e = p.communicate(timeout=300)
            assert p.returncode == 0, o + e[-4000:]
            a, b, c = o.split()
            assert (int(a), int(b), float.fromhex(c)) == (int(ok), diam, aspl)
