import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))



def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _ensure_built():
    from graphgolf_b200 import build as b
    b.build()
    import oracle
    src = oracle.reference_source()
    if not (oracle.HERE / "liboracle.so").exists() or (src is not None and src.exists() and not oracle.have_ref()):
        oracle.build()


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    _ensure_built()


@pytest.fixture(scope="session")
def gpu():
    """Skips unless a CUDA device is visible to the core library."""
    import graphgolf_b200 as g
    lib = g.load()
    if lib.ggb_device_count() < 1:
        pytest.skip("no CUDA device")
    rc = lib.ggb_init(0, 0, 0)
    assert rc == 0, g._native.last_error()
    return lib


@pytest.fixture(scope="session")
def reference_tree():
    """The reference source tree ($GGB_REFERENCE, or the one oracle/_ref was
    built from); tests that read its own data files skip without it."""
    import oracle
    src = oracle.reference_source()
    if src is None or not src.exists():
        pytest.skip("reference source tree not present (set GGB_REFERENCE)")
    return src


@pytest.fixture(scope="session")
def ref_oracle():
    import oracle
    if not oracle.have_ref():
        pytest.skip("oracle/_ref not built (reference sources were not available at build time)")
    return oracle
