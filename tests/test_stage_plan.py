"""The host staging plan (graphgolf_b200/csrc/stage_plan.h): how uploads from
pageable memory are cut into units that the staging threads copy into pinned
memory and send to the device.  Compiled with the host C++ compiler and run
on seeded random uploads (tests/stage_plan/check.cc); no GPU needed."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_stage_plan_tiles_every_upload(tmp_path):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "check"
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", str(ROOT / "graphgolf_b200" / "csrc"),
                    str(ROOT / "tests" / "stage_plan" / "check.cc"), "-o", str(exe)], check=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.startswith("ok 4000")
