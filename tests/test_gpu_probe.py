"""The roofline probes bench.py reports against: the random-row gather roof
and the L2 streaming ceiling.  Both must return a positive rate, reject bad
sizes, and order as the hardware does (bulk streaming of an L2-resident
buffer is at least as fast as register-bound random 32-byte gathers)."""
import ctypes as C

import pytest

import graphgolf_b200 as gg

pytestmark = pytest.mark.gpu


def test_probes(gpu):
    lib = gg.load()
    g, s = C.c_double(0), C.c_double(0)
    assert lib.ggb_probe_l2_gather(65536, 16, 4096, 5, C.byref(g)) == 0
    assert lib.ggb_probe_l2_stream(64, 5, C.byref(s)) == 0
    assert g.value > 100.0 and s.value > 100.0
    # the gather probe counts algorithmic bytes (adjacency + rows); its
    # physical L2 rate is somewhat below that figure
    assert s.value > 0.5 * g.value


def test_probe_bad_sizes(gpu):
    lib = gg.load()
    x = C.c_double(0)
    assert lib.ggb_probe_l2_stream(0, 5, C.byref(x)) != 0
    assert lib.ggb_probe_l2_stream(97, 5, C.byref(x)) != 0
    assert lib.ggb_probe_l2_stream(8, 0, C.byref(x)) != 0
    assert lib.ggb_probe_l2_gather(1000, 4, 100, 5, C.byref(x)) != 0
