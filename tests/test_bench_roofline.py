"""The bench line's roofline block (CPU: pure arithmetic on given figures).
The peak is the L2 streaming ceiling when the probe measured one, the
gather probe otherwise; achieved counts algorithmic bytes, and the physical
L2 and DRAM rates are reported against their own ceilings."""
import importlib.util
from pathlib import Path

import pytest

_spec = importlib.util.spec_from_file_location("bench", Path(__file__).resolve().parent.parent / "bench.py")
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def test_peak_is_the_stream_ceiling():
    r = bench.roofline("k", alg=29.0e9, ms=1.45, l2_roof=17.8e3, hbm_peak=6442.9, hbm_kind="measured",
                       traffic=1.156e9, lts=18.55e9, lts_pct=45.4, l2_stream=18.0e3)
    assert r["bound"] == "l2" and r["unit"] == "GB/s"
    assert r["achieved"] == pytest.approx(29.0e9 / 1.45e-3 / 1e9)
    assert r["peak"] == 18.0e3
    assert r["frac"] == pytest.approx(r["achieved"] / 18.0e3)
    assert r["frac_of_l2_gather_peak"] == pytest.approx(r["achieved"] / 17.8e3)
    assert r["lts_gbs"] == pytest.approx(18.55e9 / 1.45e-3 / 1e9)
    assert r["frac_of_l2_stream"] == pytest.approx(r["lts_gbs"] / 18.0e3)
    assert r["dram_frac"] == pytest.approx(1.156e9 / 1.45e-3 / 1e9 / 6442.9)
    assert "ggb_probe_l2_stream" in r["peak_source"]


def test_gather_probe_when_no_stream_figure():
    r = bench.roofline("k", alg=1e9, ms=1.0, l2_roof=10e3, hbm_peak=6442.9, hbm_kind="fallback",
                       traffic=None, lts=None)
    assert r["peak"] == 10e3 and r["frac"] == pytest.approx(0.1)
    assert "ggb_probe_l2_gather" in r["peak_source"]
    assert "dram_frac" not in r and "frac_of_l2_stream" not in r
    assert r["hbm_peak_source"].startswith("fallback")


def test_sweep_bytes_formula():
    # per dense sweep: N*d*4 (adjacency) + N*d*W/8 (gathers) + 2*N*W/8 (own row + write)
    n, d, w = 65536, 16, 4096
    assert bench.sweep_bytes(n, d, 48, w) == 48 * (n * d * 4 + n * d * w // 8 + 2 * n * w // 8)
