#!/usr/bin/env python3
"""Benchmark of the exact APSP evaluator: evaluations per second.

Default workload (N=1): one seeded random simple 16-regular graph with
N = 65536 vertices (int32 adjacency [65536][16], 4 MiB), all 65536 sources,
g = 1.  A step is one complete exact evaluation (diameter, integer distance
total, ASPL) of that graph.

* ``value``  -- evals/s with the adjacency already in HBM: the persistent
  kernel timed with CUDA events on its launching stream, the L2 flushed
  (a 512 MiB write) before every step, outside the events.
* ``e2e``    -- the same metric through the public C ABI with host buffers
  (ggb_eval_general: pinned staging, H2D of the adjacency, kernel, D2H of the
  result block, synchronise), wall-clock per call.
* ``roofline`` -- the dominant kernel (the persistent sweep kernel): its
  algorithmic bytes (per dense sweep: N*d*4 adjacency + N*d*W/8 gathered rows
  + N*W/8 own row read + N*W/8 write) over its own event-timed duration
  (events recorded by the library on the launching stream), against the
  measured HBM copy bandwidth, and against the measured random-row L2 gather
  rate (ggb_probe_l2_gather), the roof an L2-resident sweep meets.
* ``cpu_baseline`` -- the reference's own OpenMP evaluator (compiled from its
  sources into oracle/_ref) on this host's cores, over a bounded sample.

* ``batch`` -- the mixed batch (a 4096-vertex base graph and 256 single-swap
  candidates of 512..16384-vertex graphs) in one autotuned launch: graphs/s,
  e2e, roofline of the batch kernel.
* ``sa`` -- the annealing race at N=16384, d=12: wall seconds of plain device
  annealing (the reference's one-candidate step) for a fixed number of steps,
  and of the batched+learned annealer to reach the same exact distance total.

``--impl reference`` times that reference CPU evaluator alone (all host
threads) on the same workload and prints its own line.

Multi-GPU (torchrun, one process per GPU): every rank evaluates its own
seeded graph of the same size (independent objects, no collective in the data
path), timing is bracketed by barriers and the max over ranks is taken:
weak scaling.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "exact APSP evals/s (N=65536, d=16, all sources)"
UNIT = "evals/s"
WORKLOADS = {
    "n65536d16": dict(nodes=65536, degree=16, groups=1, seed=1),
    "n65536d16g16": dict(nodes=65536, degree=16, groups=16, seed=1),
    "n16384d12": dict(nodes=16384, degree=12, groups=1, seed=2),
    "n1024d8": dict(nodes=1024, degree=8, groups=1, seed=1),
}


def _env_int(name, default):
    v = os.environ.get(name)
    return int(v) if v not in (None, "") else default


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _graph(wl: dict, rank: int):
    from graphgolf_b200 import graphs
    seed = wl["seed"] + 1000 * rank
    if wl["groups"] > 1:
        return graphs.symmetric_regular(wl["nodes"], wl["degree"], wl["groups"], seed)
    return graphs.random_regular(wl["nodes"], wl["degree"], seed)


class Clocks:
    """Samples SM clocks and throttle reasons during the timed region: NVML
    read in a background thread every 10 ms (reads only; nothing is set)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.max_mhz = None
        self._stop = None
        self._thread = None
        self.err = None

    def __enter__(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report it, never invent a sample
            self.err = f"nvml unavailable: {type(e).__name__}"
            return self
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    mhz = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((mhz, rs))
                except Exception:
                    pass
                self._stop.wait(0.01)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *a):
        if self._thread:
            self._stop.set()
            self._thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [self.err or "no samples"],
                    "samples": 0}
        mhz = [m for m, _ in self.samples]
        reasons = sorted({k for _, r in self.samples for k, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(mhz)}


def sweep_bytes(nodes: int, degree: int, dense_levels: int, window_bits: int) -> int:
    """Algorithmic bytes of the persistent kernel per launch: per dense sweep,
    the adjacency (N*d*4), the d gathered rows of every vertex (N*d*W/8), its
    own row read and the new row written (2*N*W/8) -- the per-level figure of
    the bit-parallel BFS with W-bit rows."""
    row = window_bits // 8
    return dense_levels * (nodes * degree * 4 + nodes * degree * row + 2 * nodes * row)


def ball_bytes(nodes: int, degree: int, windows: int, window_bits: int) -> int:
    """Algorithmic bytes of the ball pre-pass: the 1 + d + d^2 + d^3 adjacency
    entries of every vertex's three-hop ball read, and its S_3 row of every
    window written out."""
    return nodes * (1 + degree + degree ** 2 + degree ** 3) * 4 + windows * nodes * window_bits // 8


def survey_formula_bytes(nodes: int, degree: int, levels: int, window_bits: int) -> int:
    """The same figure if every executed level were a dense sweep (the
    reference algorithm's work at this window width)."""
    row = window_bits // 8
    return levels * (nodes * degree * 4 + nodes * degree * row + 2 * nodes * row)


def _profile(workload: str) -> dict:
    """Per-launch DRAM and L2 bytes of the committed ncu captures of this
    workload (profiles/apsp_<workload>_traffic.json), or {}."""
    tp = ROOT / "profiles" / f"apsp_{workload}_traffic.json"
    return json.loads(tp.read_text()) if tp.exists() else {}


def l2_gather_roof(lib, n: int, d: int, window_bits: int):
    """The measured roof of a dense sweep: ggb_probe_l2_gather's random-row OR
    sweeps with the kernel's own access width at the same N, d and W, in GB/s
    of the sweep's algorithmic bytes (None if the probe fails)."""
    g = C.c_double(0)
    return g.value if lib.ggb_probe_l2_gather(n, d, window_bits, 20, C.byref(g)) == 0 and g.value > 0 else None


_L2_STREAM = {}


def l2_stream_roof(lib):
    """The L2 streaming ceiling (ggb_probe_l2_stream over a 64 MiB
    L2-resident buffer, the size of the headline's two window matrices) in
    GB/s, measured once per process (None if the probe fails)."""
    if "gbs" not in _L2_STREAM:
        g = C.c_double(0)
        _L2_STREAM["gbs"] = g.value if lib.ggb_probe_l2_stream(64, 10, C.byref(g)) == 0 and g.value > 0 else None
    return _L2_STREAM["gbs"]


def roofline(kernel: str, alg: float, ms: float, l2_roof, hbm_peak: float, hbm_kind: str, traffic, lts,
             lts_pct=None, l2_stream=None) -> dict:
    """Roofline of one kernel launch.  The sweeps' working set is L2-resident
    by design, so the bound is L2: `peak` is the L2 streaming ceiling measured
    live (bulk copies of an L2-resident buffer, ggb_probe_l2_stream), and the
    random-row gather probe at the same N, d and window is reported beside it.
    `achieved` counts the sweeps' algorithmic bytes; `frac_of_l2_stream` puts
    the kernel's physical L2 bytes (committed ncu capture) against the same
    ceiling.  The physical DRAM traffic is reported against the measured HBM
    copy bandwidth."""
    achieved = alg / (ms / 1e3) / 1e9
    peak = l2_stream or l2_roof
    out = {"bound": "l2", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": (achieved / peak) if peak else None, "traffic": traffic, "kernel": kernel,
           "ms_per_launch": ms, "algorithmic_bytes_per_launch": alg,
           "peak_source": ("ggb_probe_l2_stream: bulk copies of a 64 MiB L2-resident buffer into shared memory, "
                           "one CTA per SM, measured in this run (the rate at which L2 delivers bytes to the SMs)"
                           if l2_stream else
                           "ggb_probe_l2_gather: random-row OR sweeps with the kernel's own 32-byte accesses "
                           "at the same N, d and window, measured in this run"),
           "l2_gather_peak_gbs": l2_roof,
           "frac_of_l2_gather_peak": (achieved / l2_roof) if l2_roof else None,
           "hbm_peak_gbs": hbm_peak,
           "hbm_peak_source": "measured hbm_gbs (MEASURED_PEAKS.json)" if hbm_kind == "measured"
           else "fallback 6650 GB/s"}
    if traffic:
        out["dram_gbs"] = traffic / (ms / 1e3) / 1e9
        out["dram_frac"] = out["dram_gbs"] / hbm_peak
    if lts:
        out["lts_bytes_per_launch"] = lts
        out["lts_gbs"] = lts / (ms / 1e3) / 1e9
        if l2_stream:
            out["frac_of_l2_stream"] = out["lts_gbs"] / l2_stream
    if lts_pct is not None:
        out["lts_throughput_pct"] = lts_pct
    out["note"] = ("achieved counts every gather of every dense sweep (the reference algorithm's bytes), "
                   "including the parts the fullness checks and full-row stamps skip, so it can read a little "
                   "above the ceiling; frac_of_l2_stream is the physical L2 rate against it; traffic = DRAM "
                   "bytes per launch from the committed ncu capture under profiles/")
    return out


def width_sweep(lib, one, n: int, d: int, groups: int, args) -> dict:
    """The headline graph at forced source-window widths of 64, 128, 256 and
    512 bits (the reference's one-word chunk and its vector widths): evals/s
    over CUDA events on the launching stream (L2 flushed before each step),
    the persistent kernel's time, its algorithmic GB/s, and DRAM / L2 GB/s
    from the committed ncu launch list of the same widths."""
    import graphgolf_b200 as gg
    import torch
    prof = _profile(f"{args.workload}_widths")
    out = {"steps": 3, "rows": []}
    for bits in (64, 128, 256, 512):
        gg.set_tuning(bits, 0)
        one()
        lib.ggb_set_timing(1)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(3)]
        kms = []
        for e in evs:
            r = one(e)
            mb, mp = C.c_double(0), C.c_double(0)
            if lib.ggb_kernel_times(C.byref(mb), C.byref(mp)) == 0:
                kms.append(mp.value)
        lib.ggb_set_timing(0)
        torch.cuda.synchronize()
        ms = statistics.mean(a.elapsed_time(b) for a, b in evs)
        km = statistics.mean(kms) if kms else ms
        alg = sweep_bytes(n, d, r.dense_levels, r.window_bits)
        row = {"window_bits": r.window_bits, "windows": r.windows, "dense_levels": r.dense_levels,
               "evals_per_s": 1e3 / ms, "ms_per_eval": ms, "kernel_ms": km,
               "algorithmic_gbs": alg / (km / 1e3) / 1e9, "total": r.total, "diameter": r.diameter}
        pk = prof.get(str(bits), {})
        if pk.get("dram_bytes_per_launch"):
            row["dram_gbs"] = pk["dram_bytes_per_launch"] / (km / 1e3) / 1e9
        if pk.get("lts_bytes_per_launch"):
            row["l2_gbs"] = pk["lts_bytes_per_launch"] / (km / 1e3) / 1e9
        out["rows"].append(row)
    out["same_answer"] = len({(x["diameter"], x["total"]) for x in out["rows"]}) == 1
    out["traffic_source"] = ("profiles/apsp_n65536d16_widths_traffic.json (ncu launch list, one pass)"
                             if prof else None)
    return out


def g16_block(lib, hbm_peak: float, hbm_kind: str) -> dict:
    """The symmetric variant of the headline graph: 16 rotation groups
    (v <-> v + N/16), so only 4096 of the 65536 sources run; evals/s with the
    adjacency resident (L2 flushed before each step, CUDA events on the
    launching stream) and the kernel's roofline."""
    import numpy as np
    import torch
    from graphgolf_b200 import _native, graphs
    wl = WORKLOADS["n65536d16g16"]
    n, d, grp = wl["nodes"], wl["degree"], wl["groups"]
    g = graphs.symmetric_regular(n, d, grp, wl["seed"])
    adj_dev = torch.from_numpy(np.ascontiguousarray(g.adj)).cuda()
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    res = _native.ggb_result()
    lib.ggb_set_timing(1)
    evs, kms = [], []
    for k in range(13):
        e = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        with torch.cuda.stream(stream):
            flush.fill_(1)
            e[0].record(stream)
            if lib.ggb_launch_general_device(n, n // grp, grp, d, adj_dev.data_ptr(), 0, sptr):
                raise RuntimeError(_native.last_error())
            e[1].record(stream)
        if lib.ggb_collect(sptr, C.byref(res)):
            raise RuntimeError(_native.last_error())
        mb, mp = C.c_double(0), C.c_double(0)
        if k >= 3:
            evs.append(e)
            if lib.ggb_kernel_times(C.byref(mb), C.byref(mp)) == 0:
                kms.append(mp.value)
    lib.ggb_set_timing(0)
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(b) for a, b in evs)
    km = statistics.mean(kms) if kms else ms
    r = _native.ggb_result()
    alg = sweep_bytes(n, d, res.dense_levels, res.window_bits)
    kp = _profile("n65536d16g16").get("apsp_persistent_kernel", {})
    roof = roofline(f"apsp_persistent_kernel<{res.window_bits // 128}>", alg, km,
                    l2_gather_roof(lib, n, d, res.window_bits), hbm_peak, hbm_kind,
                    kp.get("dram_bytes_per_launch"), kp.get("lts_bytes_per_launch"),
                    l2_stream=l2_stream_roof(lib))
    del r
    return {"workload": "n65536d16g16: rotationally symmetric 16-regular graph, N=65536, g=16 (4096 sources)",
            "evals_per_s": 1e3 / ms, "ms_per_eval": ms, "kernel_ms": km, "window_bits": res.window_bits,
            "windows": res.windows, "dense_levels": res.dense_levels, "diameter": res.diameter,
            "total": res.total, "steps": len(evs), "roofline": roof}


def cpu_baseline(adj, budget_s: float = 12.0):
    """The reference OpenMP evaluator on this host, bounded to ~budget_s."""
    import oracle
    if not oracle.have_ref():
        return None
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    n = adj.shape[0]
    # calibrate on a 1/64 share of the source chunks (the reference's MPI split)
    t0 = time.perf_counter()
    oracle.ref_general(adj, procs=64, rank=0)
    t_share = time.perf_counter() - t0
    est_full = t_share * 64
    if est_full <= budget_s:
        k, t0 = 0, time.perf_counter()
        while True:
            oracle.ref_general(adj)
            k += 1
            if time.perf_counter() - t0 >= budget_s or k >= 50:
                break
        el = time.perf_counter() - t0
        return {"value": k / el, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"{k} full evaluation(s) of the bench graph in {el:.2f} s"}
    procs = 64
    while procs > 1 and t_share * 64 / procs * 2 <= budget_s:
        procs //= 2
    t0 = time.perf_counter()
    oracle.ref_general(adj, procs=procs, rank=0)
    el = time.perf_counter() - t0
    return {"value": (1.0 / procs) / el, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"rank 0 of {procs} (1/{procs} of the source chunks) in {el:.2f} s"}


def common_config(args, wl: dict) -> dict:
    """The `config` both arms print: the workload by name and size, the L2
    policy and the parallelism (identical strings in both arms)."""
    return {"workload": args.workload, "nodes": wl["nodes"], "degree": wl["degree"], "groups": wl["groups"],
            "seed": wl["seed"],
            "l2_policy": "GPU arm: 512 MiB flush write before every timed step, outside the events; "
                         "CPU reference arm: none (no cache to flush between full evaluations)",
            "parallelism": f"independent graph per rank x{args.gpus}"}


def run_reference_arm(args, wl):
    """The reference's own OpenMP evaluator (general/evaluation.c, compiled
    from its sources into oracle/_ref) on the same graph.  The graph is drawn
    by oracle.graphgen, a pure-Python copy of the package's generator, so this
    process loads none of the package's libraries."""
    import oracle
    from oracle import graphgen
    rank = _env_int("RANK", 0)
    if rank != 0:
        return 0
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built from the reference "
                          "sources (reference tree absent at build time)"}))
        return 0
    n, d, grp = wl["nodes"], wl["degree"], wl["groups"]
    if grp > 1:
        edges = graphgen.symmetric_regular_edges(n, d, grp, wl["seed"])
    else:
        edges = graphgen.random_regular_edges(n, d, wl["seed"])
    adj = graphgen.create_adj(n, d, edges)
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    t0 = time.perf_counter()
    oracle.ref_general(adj, procs=64, rank=0, groups=grp)
    est_full = (time.perf_counter() - t0) * 64
    # each step is one full evaluation unless that would take the whole run past ~3 minutes
    procs = 1
    while procs < 64 and est_full / procs * (args.steps + args.warmup) > 150:
        procs *= 2
    for _ in range(args.warmup):
        oracle.ref_general(adj, procs=procs, rank=0, groups=grp)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ok, diam, aspl = oracle.ref_general(adj, procs=procs, rank=0, groups=grp)
    el = time.perf_counter() - t0
    value = args.steps / procs / el
    sample = "one full evaluation per step" if procs == 1 else f"rank 0 of {procs} source-chunk shares per step"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded random regular graph)",
            "config": common_config(args, wl), "impl": "reference",
            "answer": {"diameter": diam, "aspl": aspl} if procs == 1 else None,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="n65536d16", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the mixed-batch measurement")
    ap.add_argument("--no-sa", action="store_true", help="skip the annealing race")
    ap.add_argument("--shard", action="store_true",
                    help="one graph per job, its source windows spread over the ranks (the reference's MPI "
                         "split) with a 16-byte NCCL all-reduce: strong scaling")
    ap.add_argument("--no-widths", action="store_true",
                    help="skip the window-width sweep (64..512 bits) and the g=16 symmetric graph")
    ap.add_argument("--sa-plain-steps", type=int, default=30000, help="plain annealing steps that set the target")
    ap.add_argument("--flush-mib", type=int, default=512, help="L2 flush buffer written before every step")
    ap.add_argument("--window-bits", type=int, default=0, help="force the source-window width (0 = automatic)")
    ap.add_argument("--ball", type=int, default=-1, choices=[-1, 0, 1],
                    help="ball pre-pass policy: -1 automatic, 0 never, 1 whenever feasible")
    ap.add_argument("--case", choices=["sa-step", "batch", "mlp"],
                    help="run one small case of a component for a profiler and exit")
    args = ap.parse_args()
    if args.case:
        return run_case(args.case)
    args.warmup = max(args.warmup, 3)
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, wl)

    import numpy as np
    import torch

    import graphgolf_b200 as gg
    from graphgolf_b200 import _native

    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    lib = gg.load()
    if lib.ggb_init(local, wl["nodes"], wl["degree"]) != 0:
        raise RuntimeError(_native.last_error())
    if args.shard:
        return run_sharded(args, wl, lib, rank, world, local, dist)
    if args.window_bits:
        gg.set_tuning(args.window_bits, 0)
    gg.set_ball(args.ball)

    g = _graph(wl, rank)
    n, d, groups = wl["nodes"], wl["degree"], wl["groups"]
    bn = n // groups
    adj_dev = torch.from_numpy(np.ascontiguousarray(g.adj)).cuda()
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)
    flush = torch.empty(max(args.flush_mib, 200) * 1024 * 1024, dtype=torch.uint8, device="cuda")
    res = _native.ggb_result()

    def one(timed_events=None):
        with torch.cuda.stream(stream):
            flush.fill_(1)
            if timed_events:
                timed_events[0].record(stream)
            rc = lib.ggb_launch_general_device(n, bn, groups, d, adj_dev.data_ptr(), 0, sptr)
            if rc:
                raise RuntimeError(_native.last_error())
            if timed_events:
                timed_events[1].record(stream)
        if lib.ggb_collect(sptr, C.byref(res)):
            raise RuntimeError(_native.last_error())
        return res

    for _ in range(args.warmup):
        one()
    first = gg.Result.from_c(res)
    lib.ggb_set_timing(1)
    kt_ball, kt_pers = [], []
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = lib.ggb_kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        for k in range(args.steps):
            one(evs[k])
            assert res.total == first.total and res.diameter == first.diameter
            mb, mp = C.c_double(0), C.c_double(0)
            if lib.ggb_kernel_times(C.byref(mb), C.byref(mp)) == 0:
                kt_ball.append(mb.value)
                kt_pers.append(mp.value)
        torch.cuda.synchronize()
    lib.ggb_set_timing(0)
    if dist:
        dist.barrier()
    launches = lib.ggb_kernel_launches() - launches0
    per = [a.elapsed_time(b) for a, b in evs]
    t_dev = sum(per) / 1e3
    t_max = t_dev
    if dist:
        tt = torch.tensor([t_dev], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    value = world * args.steps / t_max
    mean_ms = t_dev / args.steps * 1e3

    # e2e: the public C ABI with host buffers, H2D + kernel + D2H per call
    host_adj = np.ascontiguousarray(g.adj)
    for _ in range(2):
        gg.evaluate(host_adj, groups=groups)
    if dist:
        dist.barrier()
    h2d0 = lib.ggb_h2d_bytes()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = gg.evaluate(host_adj, groups=groups)
        assert r.total == first.total
    e2e_t = time.perf_counter() - t0
    h2d_per_step = (lib.ggb_h2d_bytes() - h2d0) // args.steps
    e2e_max = e2e_t
    if dist:
        tt = torch.tensor([e2e_t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_max = float(tt.item())
    e2e_value = world * args.steps / e2e_max

    peak, peak_kind = _peaks()
    # dominant kernel: the persistent kernel (dense sweeps); the ball pre-pass is reported beside it
    pers_ms = statistics.mean(kt_pers) if kt_pers else mean_ms
    ball_ms = statistics.mean(kt_ball) if kt_ball else 0.0
    alg = sweep_bytes(n, d, first.dense_levels, first.window_bits)
    achieved = alg / (pers_ms / 1e3) / 1e9
    l2_roof = l2_gather_roof(lib, n, d, first.window_bits)
    prof = _profile(args.workload)
    kp = prof.get("apsp_persistent_kernel", {})
    traffic = kp.get("dram_bytes_per_launch")
    lts = kp.get("lts_bytes_per_launch")

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded random regular graph, per-pair-retry pairing model)",
            "config": common_config(args, wl),
            "run": {"sources": bn, "window_bits": first.window_bits, "windows": first.windows,
                    "levels": first.levels, "dense_levels": first.dense_levels,
                    "diameter": first.diameter, "total": first.total, "aspl": first.aspl},
            "roofline": roofline(f"apsp_persistent_kernel<{first.window_bits // 128}>", alg, pers_ms, l2_roof,
                                 peak, peak_kind, traffic, lts, kp.get("lts_throughput_pct"),
                                 l2_stream_roof(lib)),
            "ball_prepass": {"ms_per_launch": ball_ms,
                             "algorithmic_bytes_per_launch": ball_bytes(n, d, first.windows, first.window_bits)
                             if ball_ms else 0,
                             "traffic": prof.get("ball_kernel", {}).get("dram_bytes_per_launch")},
            "survey_formula_bytes_per_eval": survey_formula_bytes(n, d, first.levels, first.window_bits),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d_per_step),
                    "d2h_bytes_per_step": 96, "input_bytes_per_step": n * d * 4,
                    "note": "the int32 adjacency (input bytes) crosses PCIe as 16-bit ids when every id "
                            "fits, widened on the device; h2d bytes are the library's own DMA count"},
            "gpu_launches": int(launches),
            "clocks": clk.summary()}

    if rank == 0 and world == 1 and not args.no_widths and groups == 1:
        line["widths"] = width_sweep(lib, one, n, d, groups, args)
        gg.set_tuning(args.window_bits, 0)
    if rank == 0 and world == 1 and not args.no_widths and args.workload == "n65536d16":
        line["g16"] = g16_block(lib, peak, peak_kind)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(host_adj)
    if rank == 0 and world == 1 and not args.no_ref_gpu and groups == 1:
        line["reference_cuda"] = reference_cuda(host_adj, first)
    if rank == 0 and world == 1 and not args.no_batch:
        line["batch"] = batch_bench(peak, peak_kind, lib)
    if rank == 0 and world == 1 and not args.no_sa:
        line["sa"] = sa_bench(args.sa_plain_steps)
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_sharded(args, wl, lib, rank: int, world: int, local: int, dist) -> int:
    """One evaluation of the bench graph per step with its source windows
    spread over the ranks: rank r runs windows r, r + world, ... (the
    reference's MPI split, general/evaluation.c:166) and the ranks join
    diameter and distance sum with two all-reduces of 8 and 16 bytes (NCCL;
    general/evaluation.c:247-248).  Time per step: CUDA events on the
    launching stream around the partial evaluation, the read-back and the
    all-reduces; max over ranks.  value = evaluations per second of the job
    (strong scaling: the graph does not grow with the ranks)."""
    import numpy as np
    import torch
    import graphgolf_b200 as gg
    from graphgolf_b200 import _native
    from graphgolf_b200.distributed import allreduce_partial
    n, d, groups = wl["nodes"], wl["degree"], wl["groups"]
    g = _graph(wl, 0)                       # the same graph on every rank
    adj_dev = torch.from_numpy(np.ascontiguousarray(g.adj)).cuda()
    stream = torch.cuda.Stream()
    sptr = C.c_void_p(stream.cuda_stream)
    flush = torch.empty(max(args.flush_mib, 200) * 1024 * 1024, dtype=torch.uint8, device="cuda")
    part = _native.ggb_partial()

    def step(ev=None):
        with torch.cuda.stream(stream):
            flush.fill_(1)
            if ev:
                ev[0].record(stream)
            if lib.ggb_launch_general_partial_device(n, n // groups, groups, d, adj_dev.data_ptr(), 0, rank, world,
                                                     sptr):
                raise RuntimeError(_native.last_error())
            if lib.ggb_collect_partial(sptr, C.byref(part)):
                raise RuntimeError(_native.last_error())
            if dist:
                diam, disc, total = allreduce_partial(part, device="cuda")
            else:
                diam, disc, total = part.diam, part.disconnected, part.sum
            if ev:
                ev[1].record(stream)
        return gg.finish_general(n, diam, disc, total)

    for _ in range(args.warmup):
        first = step()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.ggb_kernel_launches()
    with Clocks(local) as clk:
        for k in range(args.steps):
            r = step(evs[k])
            assert (r.diameter, r.total) == (first.diameter, first.total)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t = sum(a.elapsed_time(b) for a, b in evs) / 1e3
    t_max = t
    if dist:
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    line = {"metric": METRIC, "value": args.steps / t_max, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded random regular graph, per-pair-retry pairing model)",
            "config": {**common_config(args, wl),
                       "parallelism": f"source windows of one graph over {world} ranks, 16-byte all-reduce"},
            "run": {"diameter": first.diameter, "total": first.total, "windows_per_rank": part.windows,
                    "window_bits": part.window_bits},
            "gpu_launches": int(lib.ggb_kernel_launches() - launches0), "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def batch_bench(peak: float, peak_kind: str, lib) -> dict:
    """The mixed batch: a 4096-vertex 12-regular base graph and 256 seeded
    2-opt candidates of 12-regular graphs with 512..16384 vertices, all in one
    cooperative launch replayed from a CUDA graph, plan autotuned.  value =
    graphs per second with the adjacency resident (launch timed with CUDA
    events by the library); e2e = host arrays in, results out."""
    import graphgolf_b200 as gg
    from graphgolf_b200 import graphs
    w = graphs.batch_workload()
    adjs = [x.adj for x in w]
    b = gg.Batch([x.nodes for x in w], 12)
    b.upload(adjs)
    t0 = time.perf_counter()
    bits, team, _ = b.autotune(2)
    tune_s = time.perf_counter() - t0
    b.launch()
    res = b.collect()
    for i in (0, 1, len(w) // 2, len(w) - 1):   # spot check against the single-graph evaluator
        r = gg.evaluate(adjs[i])
        assert (r.diameter, r.total) == (res[i].diameter, res[i].total)
    ms = []
    for _ in range(10):
        b.launch()
        b.collect()
        ms.append(b.kernel_ms())
    h2d0 = lib.ggb_h2d_bytes()
    t0 = time.perf_counter()
    for _ in range(5):
        b.evaluate(adjs)
    e2e_ms = (time.perf_counter() - t0) / 5 * 1e3
    h2d = (lib.ggb_h2d_bytes() - h2d0) // 5
    kms = statistics.median(ms)
    alg = sum(sweep_bytes(x.nodes, 12, r.dense_levels, r.window_bits) for x, r in zip(w, res))
    l2 = l2_gather_roof(lib, 16384, 12, bits)
    b.close()
    roof = roofline(f"apsp_batch_kernel<{bits // 128}>", alg, kms, l2, peak, peak_kind, None, None,
                    l2_stream=l2_stream_roof(lib))
    roof["l2_gather_probe_case"] = "N=16384, d=12: the largest graphs of the batch"
    return {"workload": "4096-vertex base + 256 single-swap candidates, d=12, N log-uniform 512..16384",
            "graphs": len(w), "plan": {"window_bits": bits, "team_ctas": team, "autotune_s": tune_s},
            "value": len(w) / (kms / 1e3), "unit": "graphs/s", "ms_per_batch": kms,
            "e2e": {"value": len(w) / (e2e_ms / 1e3), "unit": "graphs/s", "ms_per_batch": e2e_ms,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 48 * len(w),
                    "input_bytes_per_step": int(sum(a.nbytes for a in adjs))},
            "roofline": roof,
            "checked": "4 graphs bit-identical to the single-graph evaluator"}


def _race(g, plain_steps: int, schedule, rows) -> dict:
    """Plain device annealing (one random 2-opt candidate per step, evaluated
    in full: the reference's step) runs plain_steps steps under `schedule`;
    its best exact (diameter, distance total) is the target.  Each annealer of
    `rows` (name, candidates K, proposals G) then runs under the same schedule
    until its current graph reaches the target (at most 90 s).  Wall seconds
    on the host clock around runs that synchronise; every final graph is
    re-evaluated in full."""
    import graphgolf_b200 as gg
    from graphgolf_b200 import graphs

    def prep(a):
        if schedule is not None:
            a.schedule(*schedule, hill_climbing=False)
        return a

    an = prep(gg.Annealer(g, 1, 1, 0, seed=1))
    st0 = an.run(0)
    t0 = time.perf_counter()
    st = an.run(plain_steps)
    t_plain = time.perf_counter() - t0
    an.close()
    out = {"start_aspl": st0.cur_aspl, "target_diameter": st.best_diam, "target_total": st.best_total,
           "target_aspl": st.best_aspl,
           "plain": {"wall_s": t_plain, "steps": st.step, "accepts": st.accepts, "evals": st.evals}}
    for name, K, G in rows:
        a = prep(gg.Annealer(g, K, G, K, seed=1))
        if G > K:
            a.predicted(0, 1)
        a.target(st.best_diam, st.best_total)
        plan = a.base_plan()
        s = a.run(0)
        t0 = time.perf_counter()
        while not s.done and time.perf_counter() - t0 < 90:
            s = a.run(10)
        el = time.perf_counter() - t0
        edges = a.edges()
        a.close()
        r = gg.evaluate(graphs.create_adj(g.nodes, g.degree, edges))
        out[name] = {"wall_s": el, "reached": bool(s.done), "steps": s.step, "accepts": s.accepts,
                     "moved_swaps": s.moved_swaps, "evals": s.evals, "final_aspl": s.cur_aspl,
                     "final_checked": (r.diameter, r.total) == (s.cur_diam, s.cur_total),
                     "candidates": K, "proposals": G, "speedup_vs_plain": t_plain / el if s.done else None,
                     "base_plan": {"team_ctas": plan[0], "teams": plan[1]}}
    return out


def reference_sa_time(g, steps: int, temp_max: float, temp_min: float):
    """The reference's own annealer (general/{main,sa,common,evaluation}.c with
    OpenMP, oracle/_ref/gg_openmp) on the same graph, all host cores: its
    `Elapse time` line (general/main.c:479) over a bounded sample of steps."""
    import re
    import subprocess
    import tempfile
    import oracle
    from graphgolf_b200 import graphs
    prog = oracle.REF_DIR / "gg_openmp"
    if not prog.exists():
        return None
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        f = os.path.join(td, "in.edges")
        graphs.write_general(f, g)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        p = subprocess.run([str(prog), "-f", f, "-M", "-s", "1", "-n", str(steps), "-w", str(temp_max),
                            "-c", str(temp_min)], cwd=td, capture_output=True, text=True, env=env, timeout=600)
    m = re.search(r"Steps: (\d+),?\s+Elapse time: ([0-9.]+) sec\. \(APSP: ([0-9.]+)", p.stdout)
    if p.returncode != 0 or not m:
        return {"error": f"rc {p.returncode}", "tail": p.stdout[-300:]}
    st, el, apsp = int(m.group(1)), float(m.group(2)), float(m.group(3))
    return {"steps": st, "elapse_s": el, "apsp_s": apsp, "s_per_step": el / max(st, 1), "cores": threads,
            "what": "reference gg_openmp (OpenMP evaluator, one MPI rank) 'Elapse time' over a bounded sample"}


def sa_bench(plain_steps: int) -> dict:
    """The learned-filter configuration on a seeded random 12-regular graph,
    N=16384: simulated annealing with the reference's Metropolis rule
    (general/sa.c:371-411) and geometric cooling from temperature 100 to
    0.0001 over the plain run's steps (general/main.c:441, sa.c:508).  Plain
    device annealing sets the target; the learned annealer (4096 proposals per
    step ranked by the online-trained network, the best 64 evaluated exactly
    against the kept base, disjoint exact improvers composed) and the same
    batched annealer without the network (64 random proposals) race to it.
    The network's own gain is batched / learned.  A second race uses hill
    climbing with the best 256 (the reference's -H rule).  The reference's own
    CPU annealer is timed on the same graph over a bounded sample of steps."""
    from graphgolf_b200 import graphs
    g = graphs.random_regular(16384, 12, 2)
    t_max, t_min = 100.0, 0.0001
    cooling = (t_min / t_max) ** (1.0 / plain_steps)
    out = {"workload": "random 12-regular, N=16384, seed 2", "plain_steps": plain_steps,
           "schedule": {"temp_max": t_max, "temp_min": t_min, "cooling_per_step": cooling}}
    sa = _race(g, plain_steps, (t_max, cooling), (("learned", 64, 4096), ("batched", 64, 64)))
    if sa["learned"]["reached"] and sa["batched"]["reached"]:
        sa["network_gain"] = sa["batched"]["wall_s"] / sa["learned"]["wall_s"]
    out["annealing"] = sa
    hill = _race(g, plain_steps, None, (("learned", 256, 4096), ("batched", 256, 256)))
    if hill["learned"]["reached"] and hill["batched"]["reached"]:
        hill["network_gain"] = hill["batched"]["wall_s"] / hill["learned"]["wall_s"]
    out["hill_climbing"] = hill
    out["filter_forward"] = filter_forward_block()
    ref = reference_sa_time(g, 100, t_max, t_min)
    if ref and "s_per_step" in ref:
        ref["extrapolated_plain_steps_s"] = ref["s_per_step"] * plain_steps
    out["reference_cpu_sa"] = ref
    return out


def filter_forward_block(rows: int = 4096, reps: int = 200) -> dict:
    """The filter network's inference forward over one step's proposals
    (4096 rows, 32 -> 256 -> 256 -> 1), device-timed with CUDA events over
    back-to-back launches, against the measured dense BF16 tensor peak."""
    import numpy as np
    import graphgolf_b200 as gg
    net = gg.FilterNet(rows, 1)
    try:
        x = np.random.default_rng(3).uniform(-1, 1, (rows, 32)).astype(np.float32)
        ms = net.time_forward(x, reps)
    finally:
        net.close()
    flops = 2.0 * rows * (32 * 256 + 256 * 256 + 256)
    out = {"kernel": "forward_tc_kernel", "rows": rows, "ms_per_launch": ms, "flops_per_launch": flops,
           "tflops": flops / (ms / 1e3) / 1e12}
    try:
        pk = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        out["peak_tflops"] = pk["bf16_tflops"]
        out["peak_source"] = "measured bf16_tflops (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        out["peak_tflops"] = 1590.0
        out["peak_source"] = "fallback 1.59 PFLOP/s"
    out["frac"] = out["tflops"] / out["peak_tflops"]
    return out


def run_case(case: str) -> int:
    """One small case of a component, for profilers (no JSON line):
    sa-step  -- 4 steps of the learned annealer, N=16384, d=12, 128 of 4096;
    batch    -- 2 launches of the mixed batch (4096-bit windows, teams of 16);
    mlp      -- the filter network: forward of 4096 rows, 2 Adam steps on 128."""
    import numpy as np
    import graphgolf_b200 as gg
    from graphgolf_b200 import graphs
    lib = gg.load()
    if lib.ggb_init(0, 0, 0) != 0:
        raise RuntimeError(gg._native.last_error())
    if case == "sa-step":
        a = gg.Annealer(graphs.random_regular(16384, 12, 2), 128, 4096, 128, seed=1)
        a.predicted(0, 1)
        st = a.run(4)
        print("sa-step", st.step, st.accepts, st.cur_total)
    elif case == "batch":
        w = graphs.batch_workload()
        b = gg.Batch([x.nodes for x in w], 12)
        b.set_plan(4096, 16)
        b.upload([x.adj for x in w])
        for _ in range(2):
            b.launch()
            r = b.collect()
        print("batch", b.kernel_ms(), r[0].total)
    else:
        net = gg.FilterNet(4096, 1)
        x = np.random.default_rng(1).uniform(-1, 1, (4096, 32)).astype(np.float32)
        y = net.forward(x)
        print("mlp", float(y[0]), net.train(x[:128], 0.5 * y[:128], 2))
    return 0


def reference_cuda(adj, want):
    """The reference's own CUDA evaluator (general/evaluation.cu, compiled for
    sm_100a into oracle/_ref) on the same GPU: the GPU bar to beat."""
    import oracle
    so = oracle.REF_DIR / "libref_general_cuda.so"
    if not so.exists():
        return None
    lib = C.CDLL(str(so))
    lib.evaluation.restype = C.c_bool
    lib.evaluation.argtypes = [C.c_int] * 5 + [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int,
                                               C.c_int]
    lib.init_matrix_dev.argtypes = [C.c_int] * 4
    lib.ref_set_ranks(0, 1)
    n, d = adj.shape
    lib.init_matrix_dev(n, d, n, 1)
    dm, asp = C.c_int(0), C.c_double(0)
    lib.evaluation(n, n, 1, n * d // 2, d, adj.ctypes.data, C.byref(dm), C.byref(asp), 0, 1)
    k, t0 = 0, time.perf_counter()
    while k < 3 or time.perf_counter() - t0 < 3.0:
        lib.evaluation(n, n, 1, n * d // 2, d, adj.ctypes.data, C.byref(dm), C.byref(asp), 0, 1)
        k += 1
        if k >= 20:
            break
    el = time.perf_counter() - t0
    lib.finalize_matrix_dev()
    return {"value": k / el, "unit": UNIT, "evals": k, "same_answer": (dm.value == want.diameter
                                                                    and asp.value == want.aspl),
            "what": "reference general/evaluation.cu built for sm_100a, host-buffer call, wall clock"}


if __name__ == "__main__":
    sys.exit(main())
