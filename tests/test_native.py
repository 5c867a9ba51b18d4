"""The C ABI libraries load and export every symbol include/*.h declares
(no GPU needed: nothing here launches a kernel)."""
import ctypes
import re
from pathlib import Path

import pytest

import graphgolf_b200 as gg
from graphgolf_b200 import _native

HEADER = Path(__file__).resolve().parent.parent / "include" / "graphgolf_b200.h"


def _declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    core = sorted(set(re.findall(r"\b(ggb_\w+)\s*\(", text)))
    return core


def test_core_exports_every_declared_function():
    lib = _native.load("core")
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


@pytest.mark.parametrize("which,names", [("general", ["evaluation", "init_matrix_dev", "finalize_matrix_dev"]),
                                         ("grid", ["evaluation"])])
def test_dropins_export_reference_names(which, names):
    lib = _native.load(which)
    for n in names:
        assert hasattr(lib, n)


def test_host_library_exports():
    lib = _native.load("host")
    for n in _native.HOST_SIGNATURES:
        assert hasattr(lib, n)


def test_version_and_device_count_without_gpu():
    lib = _native.load("core")
    assert b"sm_100a" in lib.ggb_version()
    assert lib.ggb_device_count() >= 0


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_native, "LIB_DIR", tmp_path)
    monkeypatch.setattr(_native, "_libs", {})
    with pytest.raises(_native.NativeLibraryMissing):
        _native.load("core")


def test_no_cpu_fallback_in_product():
    """The product package never imports the oracle."""
    pkg = Path(gg.__file__).resolve().parent
    for f in pkg.rglob("*.py"):
        src = f.read_text()
        assert "import oracle" not in src and "from oracle" not in src, f


def test_finish_conventions():
    """Host-side completion of reduced partials, both conventions."""
    r = gg.finish_general(10, 3, 0, 50)
    assert (r.connected, r.diameter, r.total) == (True, 3, 50 + 90) and r.aspl == 140 / 90
    r = gg.finish_general(10, 11, 0, 0)
    assert (r.connected, r.diameter) == (False, 2**31 - 1)
    lib = _native.load("core")
    p = _native.ggb_partial(4, 1, 0, 0, 0, 0)
    out = _native.ggb_result()
    assert lib.ggb_finish_grid(10, ctypes.byref(p), ctypes.byref(out)) == 0
    assert (out.connected, out.diameter) == (0, 11)


def test_checkpoint_parsing_rejects_foreign_bytes():
    """Reading a checkpoint's header is host-only: bytes that are not a
    checkpoint of this library are rejected, never interpreted."""
    import numpy as np
    lib = _native.load("core")
    n, d, g, lines = (ctypes.c_int() for _ in range(4))
    for blob in (b"", b"\x00" * 16, bytes(range(256)) * 8):
        assert lib.ggb_sa_checkpoint_info(blob, len(blob), ctypes.byref(n), ctypes.byref(d), ctypes.byref(g),
                                          ctypes.byref(lines)) != 0
        e = np.empty(16, dtype=np.int32)
        assert lib.ggb_sa_checkpoint_edges(blob, len(blob), 0, e.ctypes.data) != 0
    with pytest.raises(gg.EvaluationError):
        gg.checkpoint_graph(b"\x31\x47\x47\x43" + b"\x00" * 60)


def test_every_declared_function_has_a_binding():
    """Every ggb_* function the header declares has a ctypes signature in the
    package's binding table, so Python callers never fall back to ctypes'
    default int/pointer guesses."""
    names = _declared()
    missing = [n for n in names if n not in _native.CORE_SIGNATURES]
    assert not missing, missing
