"""In-tree build of the graphgolf_b200 native libraries.

Outputs (all under graphgolf_b200/_lib/, git-ignored, shipped with the tree):

* ``libgraphgolf_b200.so`` -- the core: CUDA kernels for sm_100a and the
  ``ggb_*`` C ABI (include/graphgolf_b200.h).
* ``libgg_general.so`` / ``libgg_grid.so`` -- drop-in replacements for the
  reference's general and grid ``evaluation()`` (link-compatible C ABI);
  ``libgg_general_nr.so`` / ``libgg_grid_nr.so`` the same for its
  non-regular variants.
* ``libggb_host.so`` -- host C utilities: seeded generators, edge files,
  adjacency, checks.

nvcc cross-compiles for sm_100a without a GPU, so this runs anywhere the CUDA
toolkit is installed.  Rebuilds only what is older than its sources.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "_lib"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]
CC_FLAGS = ["-std=gnu11", "-O3", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build graphgolf_b200")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError(f"build step failed ({proc.returncode}): {' '.join(cmd)}")


def core_sources() -> list[Path]:
    return [*sorted(CSRC.glob("*.cu")), *sorted(CSRC.glob("*.cuh")), *sorted(CSRC.glob("*.h")),
            INCLUDE / "graphgolf_b200.h"]


def build(verbose: bool = False) -> dict[str, Path]:
    """Builds every native library of the package; returns their paths."""
    LIB.mkdir(exist_ok=True)
    nvcc = _nvcc()
    out: dict[str, Path] = {}

    core = LIB / "libgraphgolf_b200.so"
    cu = [p for p in sorted(CSRC.glob("*.cu"))]
    if _stale(core, core_sources()):
        objs = []
        for src in cu:
            obj = LIB / (src.stem + ".o")
            _run([nvcc, *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)])
            objs.append(str(obj))
        _run([nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(core), *objs, "-lcudart_static",
              "-lrt", "-ldl", "-lpthread"])
        for o in objs:
            Path(o).unlink(missing_ok=True)
    out["core"] = core

    for name, src in (("general", "dropin_general.c"), ("grid", "dropin_grid.c"),
                      ("general_nr", "dropin_general_nonregular.c"), ("grid_nr", "dropin_grid_nonregular.c")):
        so = LIB / f"libgg_{name}.so"
        deps = [CSRC / src, INCLUDE / "graphgolf_b200.h", core]
        if _stale(so, deps):
            _run(["gcc", *CC_FLAGS, "-shared", "-o", str(so), str(CSRC / src), f"-L{LIB}", "-lgraphgolf_b200",
                  "-Wl,-rpath,$ORIGIN"])
        out[name] = so

    host = LIB / "libggb_host.so"
    hsrc = CSRC / "host" / "graph_host.c"
    if _stale(host, [hsrc]):
        _run(["gcc", *CC_FLAGS, "-shared", "-o", str(host), str(hsrc)])
    out["host"] = host
    if verbose:
        for k, v in out.items():
            print(f"{k}: {v}")
    return out


if __name__ == "__main__":
    build(verbose=True)
