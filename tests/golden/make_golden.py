"""Generates tests/golden/apsp_golden.json: known answers of the REFERENCE's
own evaluator (compiled from its sources into oracle/_ref by oracle/Makefile)
on seeded graphs.

Each case names its graph by (generator, parameters, seed); the graph itself
is rebuilt at test time by graphgolf_b200.graphs, whose generators are
deterministic on every machine, and its adjacency hash is stored so that a
change of generator cannot silently change the answers.  The expected values
are what the reference's evaluation() returns and writes; `total` is the
exact integer the reference divides, recovered as round(ASPL * N * (N-1))
(exact: the quotient carries a relative error of at most 2^-53).

Run from the repository root:  python tests/golden/make_golden.py
(needs oracle/_ref, i.e. the reference sources at build time).
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from graphgolf_b200 import graphs  # noqa: E402

OUT = Path(__file__).resolve().parent / "apsp_golden.json"


def adj_hash(adj: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(adj, dtype=np.int32).tobytes()).hexdigest()[:16]


def build_case(c: dict):
    """Returns (adjacency, rotate_hash or None) for a case description."""
    k, p = c["kind"], c["params"]
    if k == "random":
        return graphs.random_regular(p["n"], p["d"], c["seed"]).adj, None
    if k == "symmetric":
        return graphs.symmetric_regular(p["n"], p["d"], p["g"], c["seed"]).adj, None
    if k == "union":   # two disjoint random regular graphs: disconnected
        a = graphs.random_regular(p["n"], p["d"], c["seed"]).adj
        b = graphs.random_regular(p["n"], p["d"], c["seed"] + 1).adj + p["n"]
        return np.concatenate([a, b]).astype(np.int32), None
    if k == "grid":
        g = graphs.grid_regular(p["w"], p["h"], p["d"], p["r"], c["seed"])
        rh = graphs.rotate_hash(g.nodes, p["h"], p["w"], c.get("groups", 1))
        return g.adj, rh
    raise ValueError(k)


CASES = []


def add(kind, seed, groups=1, ac=0, **params):
    CASES.append({"kind": kind, "seed": seed, "groups": groups, "added_centers": ac, "params": params})


# general, g = 1
for n, d, s in [(10, 3, 1), (16, 3, 2), (16, 4, 3), (32, 4, 4), (64, 5, 5), (100, 6, 6), (127, 8, 7),
                (128, 7, 8), (129, 4, 9), (255, 6, 10), (256, 10, 11), (257, 8, 12), (500, 10, 13),
                (1000, 3, 14), (1024, 8, 1), (2000, 12, 2), (4096, 12, 3), (5000, 30, 4)]:
    add("random", s, n=n, d=d)
# general, symmetric groups
for n, d, g, s in [(256, 6, 2, 1), (256, 6, 4, 2), (256, 8, 8, 3), (256, 8, 16, 4), (512, 4, 2, 5),
                   (1728, 30, 144, 6), (1728, 30, 16, 7), (4096, 12, 16, 8), (6000, 10, 3, 9)]:
    add("symmetric", s, groups=g, n=n, d=d, g=g)
# added centres: the last `ac` vertices are centres, based_nodes = (n-ac)/g
for n, d, g, ac, s in [(130, 6, 1, 2, 1), (134, 8, 2, 6, 2), (1040, 8, 16, 16, 3), (300, 5, 3, 30, 4),
                       (4000, 7, 5, 100, 5)]:
    add("random", s, groups=g, ac=ac, n=n, d=d)
# disconnected
for n, d, s in [(16, 3, 1), (64, 4, 2), (600, 6, 3)]:
    add("union", s, n=n, d=d)
# grid, g = 1 and rotation relabels
for w, h, d, r, g, s in [(5, 4, 4, 2, 1, 1), (10, 10, 4, 3, 1, 2), (20, 20, 4, 3, 1, 3), (10, 10, 6, 3, 1, 4),
                         (30, 20, 8, 4, 1, 5), (100, 100, 4, 3, 1, 1), (20, 20, 4, 3, 2, 6),
                         (20, 20, 6, 3, 4, 7), (64, 64, 4, 3, 4, 8)]:
    add("grid", s, groups=g, w=w, h=h, d=d, r=r)
# large (bench workloads and their symmetric variant)
add("random", 2, n=16384, d=12)
add("random", 1, n=65536, d=16)
add("symmetric", 1, groups=16, n=65536, d=16, g=16)


def expected(c: dict, adj: np.ndarray, rh) -> dict:
    n = adj.shape[0]
    g, ac = c["groups"], c["added_centers"]
    if c["kind"] == "grid":
        height = c["params"]["h"]
        ok, diam, aspl = oracle.ref_grid(adj, rh, groups=g, height=height, based_height=height // (2 if g > 1 else 1))
    else:
        ok, diam, aspl = oracle.ref_general(adj, based_nodes=(n - ac) // g, groups=g, added_centers=ac)
    out = {"connected": ok, "diameter": diam}
    if ok:
        out["aspl_hex"] = float(aspl).hex()
        out["total"] = int(round(aspl * n * (n - 1)))
    else:
        out["aspl_hex"] = float(aspl).hex() if aspl is not None else None
        out["total"] = 0
    return out


def main() -> None:
    if not oracle.have_ref():
        oracle.build()
    if not oracle.have_ref():
        raise SystemExit("oracle/_ref is not built: set GGB_REFERENCE to the reference source tree")
    rows = []
    for c in CASES:
        adj, rh = build_case(c)
        row = dict(c)
        row["nodes"] = int(adj.shape[0])
        row["degree"] = int(adj.shape[1])
        row["adj_sha"] = adj_hash(adj)
        row["expected"] = expected(c, adj, rh)
        rows.append(row)
        print(c["kind"], c["params"], c["groups"], c["added_centers"], row["expected"], flush=True)
    OUT.write_text(json.dumps({"generator": "tests/golden/make_golden.py",
                               "checker": "reference evaluator compiled from its sources (oracle/_ref)",
                               "cases": rows}, indent=1))
    print(f"wrote {OUT} ({len(rows)} cases)")


if __name__ == "__main__":
    main()
