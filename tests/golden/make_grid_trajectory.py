"""Generates tests/golden/grid_trajectory_w100h100d4r3.json: the reference's
own grid annealer (grid/{main,sa,common,evaluation,timer}.c, compiled from its
sources into oracle/_ref/gg_grid_openmp by oracle/Makefile) run for the full
grid configuration -- a seeded 100 x 100 lattice graph of degree 4 with edge
length limit 3 (graphgolf_b200.graphs.grid_regular(100, 100, 4, 3, 1)),
100 000 annealing steps, seed 1 -- on the CPU, once.

The fixture keeps the run's progress table (every row the program prints:
step, temperature, current/best ASPL and diameter, accept rate -- the
accept/reject trajectory at the program's own sampling), its final result
lines, and the SHA-256 of the edge file it writes with -o.  A GPU test runs
the same program linked against libgg_grid.so and must reproduce all three.
Lines that carry wall-clock times, host names or file names are dropped by
stable_lines(), the one filter both sides use.

Run from the repository root (it takes about an hour on 8 cores):
    python tests/golden/make_grid_trajectory.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "grid_trajectory_w100h100d4r3.json"

# The configuration: lattice width/height, degree, length limit, generator
# seed, annealing seed and steps.
CONFIG = {"width": 100, "height": 100, "degree": 4, "length": 3, "graph_seed": 1, "sa_seed": 1, "steps": 100000}

_DROP = ("Run on", "sec", "---", "Seed", "Num. of threads", "Threads", "Processes", "Num. of processes",
         "Output filename", "Input filename")


def stable_lines(text: str) -> list[str]:
    """Output lines of the reference program that do not depend on the host,
    the clock or the file names."""
    out = []
    for line in text.splitlines():
        if any(k in line for k in _DROP):
            continue
        if line[:3] in ("Mon", "Tue", "Wed", "Thu", "Fri", "Sat", "Sun"):
            continue
        out.append(line.rstrip())
    return out


def program_args(edges_in: str, edges_out: str) -> list[str]:
    c = CONFIG
    return ["-f", edges_in, "-R", str(c["length"]), "-s", str(c["sa_seed"]), "-n", str(c["steps"]), "-o", edges_out]


def write_input(path: str) -> None:
    from graphgolf_b200 import graphs
    c = CONFIG
    g = graphs.grid_regular(c["width"], c["height"], c["degree"], c["length"], c["graph_seed"])
    graphs.write_grid(path, g)


def main() -> None:
    import oracle
    prog = oracle.REF_DIR / "gg_grid_openmp"
    if not prog.exists():
        raise SystemExit("oracle/_ref/gg_grid_openmp is not built (set GGB_REFERENCE and run oracle.build())")
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.edges"), os.path.join(td, "out.edges")
        write_input(fin)
        in_sha = hashlib.sha256(Path(fin).read_bytes()).hexdigest()
        t0 = time.time()
        p = subprocess.run([str(prog), *program_args(fin, fout)], cwd=td, capture_output=True, text=True)
        wall = time.time() - t0
        if p.returncode != 0:
            raise SystemExit(f"reference program failed ({p.returncode}):\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
        out_sha = hashlib.sha256(Path(fout).read_bytes()).hexdigest()
    lines = stable_lines(p.stdout)
    OUT.write_text(json.dumps({
        "what": "reference grid annealer (gg_grid_openmp) on the seeded 100x100 d4 r3 lattice graph",
        "config": CONFIG,
        "input_sha256": in_sha,
        "output_sha256": out_sha,
        "lines": lines,
        "cpu_wall_s": round(wall, 1),
        "cpu_threads": os.environ.get("OMP_NUM_THREADS", str(os.cpu_count())),
    }, indent=1) + "\n")
    print(f"wrote {OUT} ({len(lines)} lines, {wall:.0f} s)")


if __name__ == "__main__":
    main()
