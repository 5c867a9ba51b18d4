"""The allocation-free entry point, ggb_eval_general_noalloc.

It serves callers that cannot let a library call cudaMalloc (device memory
owned by another allocator, or an annealing loop that must not allocate): the
kernel's scratch lives in a fixed 16 MiB device array inside the library.
Called through the C ABI on device-resident adjacency, it must return exactly
what the allocating device entry point returns, on two calls in a row (the
shared array keeps the previous call's contents), and it must reject a graph
too large for its array.  This file is collected last so that a failure here
leaves every other test already run; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import graphgolf_b200 as gg
import oracle
from graphgolf_b200 import _native, graphs

pytestmark = pytest.mark.gpu


def _fields(r):
    return (r.connected, r.diameter, r.aspl, r.total, r.levels, r.windows)


@pytest.mark.parametrize("n,d,g,ac,seed", [(3000, 8, 1, 0, 1), (20000, 12, 1, 0, 2), (4100, 6, 4, 4, 3),
                                           (778, 5, 1, 0, 4)])
def test_no_alloc_matches_device_entry(gpu, n, d, g, ac, seed):
    import torch
    lib = gg.load()
    adj = graphs.random_regular(n, d, seed).adj
    adj_dev = torch.from_numpy(np.ascontiguousarray(adj)).cuda()
    torch.cuda.synchronize()
    bn = (n - ac) // g
    want = oracle.general(adj, groups=g, added_centers=ac)   # the CPU restatement of the reference
    ref = _native.ggb_result()
    assert lib.ggb_eval_general_device(n, bn, g, d, adj_dev.data_ptr(), ac, None, C.byref(ref)) == 0, \
        _native.last_error()
    for _ in range(2):
        out = _native.ggb_result()
        rc = lib.ggb_eval_general_noalloc(n, bn, g, d, adj_dev.data_ptr(), ac, None, C.byref(out))
        assert rc == 0, lib.ggb_noalloc_last_error()
        # integers bit-exact, ASPL the identical double (the tolerance of every parity test here)
        assert (out.connected, out.diameter, out.total) == (ref.connected, ref.diameter, ref.total)
        assert out.aspl == ref.aspl
        assert (bool(out.connected), out.diameter, out.aspl, out.total) == want


def test_no_alloc_rejects_too_large(gpu):
    import torch
    lib = gg.load()
    assert lib.ggb_noalloc_scratch_bytes() == 16 << 20
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = _native.ggb_result()
    rc = lib.ggb_eval_general_noalloc(1 << 20, 1 << 20, 1, 4, dummy.data_ptr(), 0, None, C.byref(out))
    assert rc == -1
    assert b"too large" in lib.ggb_noalloc_last_error()
    # few enough vertices for the array, but more adjacency entries than an int32 offset reaches
    rc = lib.ggb_eval_general_noalloc(200000, 200000, 1, 20000, dummy.data_ptr(), 0, None, C.byref(out))
    assert rc == -1
    assert b"int32" in lib.ggb_noalloc_last_error()
