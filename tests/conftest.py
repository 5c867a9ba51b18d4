import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

REFERENCE = Path(os.environ.get("GGB_REFERENCE", "/root/reference"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _ensure_built():
    from graphgolf_b200 import build as b
    b.build()
    import oracle
    if not (oracle.HERE / "liboracle.so").exists() or (REFERENCE.exists() and not oracle.have_ref()):
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
    if not REFERENCE.exists():
        pytest.skip("reference source tree not present")
    return REFERENCE


@pytest.fixture(scope="session")
def ref_oracle():
    import oracle
    if not oracle.have_ref():
        pytest.skip("oracle/_ref not built (reference sources were not available at build time)")
    return oracle
