"""Host staging of the adjacency (graphgolf_b200/csrc/stage.cu): the
pageable array is copied into pinned memory by a pool of host threads and
sent to the device, as 16-bit ids when every id fits.  These tests check the
bytes that cross PCIe (the library's own DMA count) and that every thread
count and both id widths give the same answers as the oracle."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import graphgolf_b200 as gg
import oracle
from graphgolf_b200 import graphs

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def _sent(fn):
    lib = gg.load()
    b0 = lib.ggb_h2d_bytes()
    out = fn()
    return out, lib.ggb_h2d_bytes() - b0


def test_ids_cross_as_16_bits_when_they_fit(gpu):
    adj = graphs.random_regular(1024, 8, 3).adj
    r, sent = _sent(lambda: gg.evaluate(adj))
    assert sent == 1024 * 8 * 2
    assert (r.connected, r.diameter, r.aspl, r.total) == oracle.general(adj)
    # an id past 16 bits: the upload falls back to plain ints (and the device rejects the id)
    bad = adj.copy()
    bad[5, 1] = 1 << 17
    with pytest.raises(gg.EvaluationError):
        _sent(lambda: gg.evaluate(bad))


def test_graphs_above_65536_vertices_send_ints(gpu):
    """Past 65536 vertices ids need 17 bits: the ints go as they are.  The
    answer equals the device-pointer entry point's, which stages nothing."""
    import ctypes as C
    import torch
    gr = graphs.random_regular(65538, 4, 7)
    r, sent = _sent(lambda: gg.evaluate(gr.adj))
    assert sent == 65538 * 4 * 4
    assert r.connected
    lib = gg.load()
    d = torch.from_numpy(np.ascontiguousarray(gr.adj)).cuda()
    from graphgolf_b200 import _native
    ref = _native.ggb_result()
    assert lib.ggb_eval_general_device(65538, 65538, 1, 4, d.data_ptr(), 0, None, C.byref(ref)) == 0
    assert (ref.diameter, ref.total) == (r.diameter, r.total)


def test_batch_upload_bytes(gpu):
    sizes = [512, 1000, 2048, 4096]
    a = [graphs.random_regular(n, 12, n + 1).adj for n in sizes]
    with gg.Batch(sizes, 12) as b:
        res, sent = _sent(lambda: b.evaluate(a))
    assert sent == sum(n * 12 for n in sizes) * 2   # every N*12 is a multiple of 4: no padding
    for x, r in zip(a, res):
        assert (r.connected, r.diameter, r.aspl, r.total) == oracle.general(x)


_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import graphgolf_b200 as gg
from graphgolf_b200 import graphs
out = []
for n, d, s in ((1000, 6, 1), (40000, 8, 2), (3000, 6, 3)):
    r = gg.evaluate(graphs.random_regular(n, d, s).adj)
    out.append([r.diameter, r.total])
sizes = [600, 2000, 5000]
with gg.Batch(sizes, 10) as b:
    out.append([[r.diameter, r.total] for r in b.evaluate([graphs.random_regular(n, 10, n).adj for n in sizes])])
print(json.dumps(out))
"""


def test_thread_counts_and_id_widths_agree(gpu):
    """1, 2 and 7 staging threads, 16-bit ids on and off: identical answers,
    equal to the oracle's for the small graphs."""
    runs = {}
    for threads in ("1", "2", "7"):
        for narrow in ("0", "1"):
            env = dict(os.environ, GGB_STAGE_THREADS=threads, GGB_STAGE_NARROW=narrow)
            p = subprocess.run([sys.executable, "-c", _CHILD, str(ROOT)], env=env, capture_output=True, text=True,
                               timeout=600)
            assert p.returncode == 0, p.stderr[-2000:]
            runs[(threads, narrow)] = json.loads(p.stdout.strip().splitlines()[-1])
    first = next(iter(runs.values()))
    assert all(v == first for v in runs.values()), runs
    for (n, d, s), got in zip(((1000, 6, 1), (3000, 6, 3)), (first[0], first[2])):
        want = oracle.general(graphs.random_regular(n, d, s).adj)
        assert [want[1], want[3]] == got
