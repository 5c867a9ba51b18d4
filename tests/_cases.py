"""Shared helpers: the golden cases and graph rebuilding for the tests."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))
GOLDEN = ROOT / "tests" / "golden" / "apsp_golden.json"


def golden_cases():
    return json.loads(GOLDEN.read_text())["cases"]


def case_id(c) -> str:
    p = "-".join(f"{k}{v}" for k, v in c["params"].items())
    return f"{c['kind']}-{p}-g{c['groups']}-v{c['added_centers']}-s{c['seed']}"


def build(c):
    from make_golden import adj_hash, build_case
    adj, rh = build_case(c)
    assert adj_hash(adj) == c["adj_sha"], "generator drift: the seeded graph changed"
    return adj, rh


def aspl_of(c) -> float | None:
    h = c["expected"]["aspl_hex"]
    return None if h is None else float.fromhex(h)


def union_graph(n, d, seed):
    from graphgolf_b200 import graphs
    a = graphs.random_regular(n, d, seed).adj
    b = graphs.random_regular(n, d, seed + 1).adj + n
    return np.concatenate([a, b]).astype(np.int32)
