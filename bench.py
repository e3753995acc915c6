#!/usr/bin/env python
"""Benchmark: derived tuples/s of the semi-naive fixpoint on B200.

Workload (default): the Trop multi-source shortest-path program

    dist(S,Y) :- src(S), edge(S,Y).
    dist(S,Z) :- dist(S,Y), edge(Y,Z).        (min-plus)

on a seeded R-MAT scale-20 graph (1,048,576 node ids, 8,388,608 distinct
directed edges, a=0.57 b=c=0.19), i64 weights U[1,100], 64 sources.  One
step = the whole fixpoint from the resident EDB to the final `dist`
relation.  metric = |dist| / device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs its own instance (its own graph seed and
sources; no data-path collective) and `value` sums tuples over ranks divided
by the max rank time ("scaling": "weak"); with --shard the ranks split one
instance instead ("scaling": "strong"): its independent units (sources,
batch instances, query targets, triangle source vertices), or for the Bool
closure its path rows, whose Δ' rows meet in an all-gather every round.
`--impl reference` times the
reference interpreter's algorithm (the CPU restatement in oracle/, nested
loop `solve`, one thread like the reference) on complete fixpoints of a
scaled-down instance of the same distribution, one per step, and reports the
power-law fit over several sizes that extrapolates it to the full workload.
Our arm adds, on rank 0 at N = 1, the same fit extrapolated to the measured
result size (`cpu_baseline`), a fast all-core C++ baseline at the full size
(`cpu_fast`) and a check of the engine's result against it (`check`).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT / "strata-k_b200"), str(ROOT / "oracle")]

import numpy as np  # noqa: E402

METRIC = "derived tuples/s (Trop MSSP fixpoint, |dist| / device time)"
UNIT = "tuples/s"
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["mssp", "tc", "tri", "batch", "prov"], default="mssp",
                    help="mssp: the headline Trop program; tc / tri / batch: the Bool closure, triangle-count "
                         "and batched-reachability configs")
    ap.add_argument("--instances", type=int, default=4096, help="batch: number of instances")
    ap.add_argument("--queries", type=int, default=1024, help="prov: number of ?grad query pairs")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: split one workload across the ranks (mssp sources, batch instances, prov "
                         "query targets, triangle source vertices; tc path rows with the Δ' rows all-gathered "
                         "every round) instead of running a replica per rank")
    ap.add_argument("--plan", choices=["auto", "sort-merge", "dense"], default="auto")
    ap.add_argument("--tuned", action="store_true", help="apply the autotuner's cached knob values")
    ap.add_argument("--scale", type=int, default=None, help="R-MAT scale (mssp: 20, tri: 22)")
    ap.add_argument("--sources", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sort-plan", action="store_true", help="skip the sort-merge plan measurement")
    ap.add_argument("--out", default=None, help="also write the JSON line here")
    args = ap.parse_args()
    if args.scale is None:
        args.scale = 22 if args.workload == "tri" else 20
    return args


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_for(rank: int, scale: int, n_sources: int, kind: str = "mssp"):
    from strata_b200 import gen
    if kind == "tc":
        return gen.tc_workload(seed=1 + 1000 * rank)
    if kind == "tri":
        return gen.triangle_workload(scale=scale, seed=3 + 1000 * rank)
    if kind == "prov":
        return gen.prov_workload(n_queries=n_sources, seed=5 + 1000 * rank)
    if kind == "batch":
        return gen.batch_tc_workload(n_inst=n_sources, seed=4 + 1000 * rank, workers=min(16, os.cpu_count() or 1))
    return gen.mssp_workload(scale=scale, n_sources=n_sources, seed=2 + 1000 * rank)


PLANS = {"auto": 0, "sort-merge": 1, "dense": 2}


def units_arg(args) -> int:
    return {"batch": args.instances, "prov": args.queries}.get(args.workload, args.sources)


def unit_for(kind: str) -> str:
    return "queries/s" if kind == "prov" else UNIT


def metric_for(kind: str) -> str:
    return {"mssp": METRIC,
            "tc": "derived tuples/s (Bool transitive-closure fixpoint, |path| / device time)",
            "tri": "derived tuples/s (WCOJ triangle pattern count, triangles / device time)",
            "batch": "derived tuples/s (batched Bool reachability, sum of |path| over instances / device time)",
            "prov": "?grad/s (Prov_k(8) capture + exact circuits + FP32 forward/adjoint, queries / time)"}[kind]


def config(args, world):
    sharded = bool(args.shard and world > 1 and args.workload in ("mssp", "tc", "batch", "prov", "tri"))
    common = {"parallelism": f"sharded{world}" if sharded else f"replicas{world}", "plan": args.plan,
              "l2": "flushed (256 MiB write) before every timed step"}
    if args.workload == "tc":
        return {"workload": "bool_tc_er_10000n_50000e",
                "program": "path(X,Y) :- edge(X,Y). path(X,Z) :- edge(X,Y), path(Y,Z).",
                "graph": "Erdos-Renyi directed, 10,000 nodes, 50,000 distinct edges, no self-loops", **common}
    if args.workload == "prov":
        return {"workload": f"prov_reach_er_20000n_80000e_{args.queries}q_k8",
                "program": "path(X,Y) :- edge(X,Y). path(X,Z) :- edge(X,Y), path(Y,Z). (path: Prov_k(8), "
                           "edge: probabilistic)",
                "graph": "Erdos-Renyi directed, 20,000 nodes, 80,000 edges, p ~ Beta(2,5) as fp32",
                "queries": args.queries, **common}
    if args.workload == "batch":
        return {"workload": f"batch_tc_{args.instances}x_er_n100_50000_deg2_8",
                "program": "path(X,Y) :- edge(X,Y). path(X,Z) :- edge(X,Y), path(Y,Z). (per instance)",
                "graph": f"{args.instances} directed ER instances, nodes log-uniform in [100, 50000], mean "
                         "out-degree uniform in [2, 8], seeded per instance",
                "instances": args.instances, **common}
    if args.workload == "tri":
        return {"workload": f"wcoj_triangles_rmat{args.scale}",
                "program": "n(count<X>) :- e(X,Y), e(Y,Z), e(X,Z).",
                "graph": f"undirected R-MAT scale {args.scale}, {16 << args.scale} edges drawn, "
                         "deduplicated, oriented by degree", **common}
    return {
        "workload": f"trop_mssp_rmat{args.scale}_{args.sources}src",
        "program": "dist(S,Y) :- src(S), edge(S,Y). dist(S,Z) :- dist(S,Y), edge(Y,Z). (Trop)",
        "graph": f"R-MAT scale {args.scale}, {8 << args.scale} distinct directed edges, "
                 "a=0.57 b=0.19 c=0.19, i64 weights U[1,100]",
        "sources": args.sources, **common,
    }


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per launch of
# the dominant kernel, from one ncu capture of the named workload (the 16
# k_expand_dense launches of one MSSP R-MAT-20 fixpoint: 3.57 GB in total, so
# 223 MB per launch against 550 MB of algorithmic bytes — the index probes hit
# in L2); absent (null) when no capture of that workload and kernel exists.
TRAFFIC: dict = {("mssp", "k_expand_dense"): 223_022_176}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (read-only queries)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU baselines
# The reference interpreter is single-threaded (no threads, rayon or async in
# crates/strata-eval or crates/strata-cli) and its join is a nested loop,
# O(|E|·|Δ|) per round (crates/strata-eval/src/seminaive.rs:215-277): at the
# full sizes it runs for days.  Its restatement (oracle/, same algorithm) is
# therefore timed on complete fixpoints of scaled-down instances of the same
# distribution, one thread, and the time is extrapolated to the full size by
# a fitted power law  t = a · E^b  over the edge count E.

def _interp_point(kind: str, size):
    """One complete fixpoint of the restated interpreter (1 thread) on a
    scaled-down instance: returns (edges, tuples, seconds)."""
    import time as _t

    import oracle as O
    from strata_b200 import gen
    if kind == "mssp":
        w = gen.mssp_workload(scale=size, n_sources=64, seed=2)
        prog, head = O.mssp_program(w.sources, w.src, w.dst, w.w, w.source_w), "dist"
    elif kind == "tc":
        s, d = gen.er_directed(size, 5 * size, 1)
        w = gen.Workload("er", s, d)
        prog, head = O.tc_program(s, d), "path"
    elif kind == "tri":
        w = gen.triangle_workload(scale=size, edge_factor=16, seed=3)
        prog = O.count_program(w.src, w.dst)
        t0 = _t.perf_counter()
        db, _ = prog.run(semi_naive=True, threads=1)
        secs = _t.perf_counter() - t0
        return len(w.src), int(db["ntri"][0][0][0][1]) if db["ntri"] else 0, secs
    else:
        raise ValueError(kind)
    sess = O.Session(prog)
    counts, _, secs = sess.run(threads=1)
    sess.close()
    return len(w.src), counts[head], secs


# Scaled-down sizes of each workload: R-MAT scale (mssp, tri) or ER node count
# at mean out-degree 5 (tc); together about 10-20 s of single-core time.
INTERP_SIZES = {"mssp": (6, 7, 8, 9), "tc": (150, 200, 300, 400), "tri": (6, 7, 8)}
# The bounded sample one reference-arm step runs (a complete fixpoint).
INTERP_STEP = {"mssp": 8, "tc": 300, "tri": 7}


def _fit(points):
    """Least-squares fit of log t = log a + b log E over the points."""
    e = np.log([p[0] for p in points])
    t = np.log([max(p[2], 1e-9) for p in points])
    b, loga = np.polyfit(e, t, 1)
    return float(np.exp(loga)), float(b)


def _size_words(kind: str) -> str:
    return {"mssp": "R-MAT scales, 64 sources,", "tc": "ER node counts at mean out-degree 5:",
            "tri": "undirected R-MAT scales, edge factor 16,"}.get(kind, "sizes")


def interp_extrapolation(kind: str, full_edges: int, full_tuples: int):
    """The restated interpreter on complete fixpoints at INTERP_SIZES, fitted
    and extrapolated to the full workload."""
    pts = [_interp_point(kind, sz) for sz in INTERP_SIZES[kind]]
    a, b = _fit(pts)
    secs = a * float(full_edges) ** b
    return {"value": full_tuples / secs if secs > 0 else 0.0, "unit": UNIT, "cores": 1, "kind": "port",
            "extrapolated": True,
            "sample": (f"restated reference interpreter (single-threaded nested-loop semi-naive, as "
                       f"strata run --semi-naive) on complete fixpoints of scaled-down instances "
                       f"({_size_words(kind)} {list(INTERP_SIZES[kind])}); fitted t = a*E^b with b = {b:.2f}, "
                       f"extrapolated to E = {full_edges} edges and {full_tuples} tuples: {secs:.3e} s "
                       f"(extrapolated)"),
            "points": [{"edges": int(p[0]), "tuples": int(p[1]), "seconds": round(p[2], 4)} for p in pts],
            "exponent": b, "extrapolated_seconds": secs}


def interp_units(kind: str, wl, budget_s: float = 20.0):
    """Batch and prov: the restated reference algorithm, one thread, on whole
    units (instances smallest first; queries in order) until `budget_s`.  The
    rate covers the units run; for batch the per-instance time is also fitted
    against the edge count and summed over all instances (extrapolated)."""
    import time as _t

    import oracle as O
    if kind == "prov":
        t0 = _t.time()
        done = 0
        for q in range(len(wl.qs)):
            proofs, _ = O.prov_tc(wl.n, wl.src, wl.dst, wl.p64, 8, wl.qs[q:q + 1], wl.qt[q:q + 1], threads=1)
            O.compile_grad(proofs[0], wl.p64)
            done += 1
            if _t.time() - t0 > budget_s:
                break
        secs = _t.time() - t0
        return {"value": done / secs, "unit": "queries/s", "cores": 1, "kind": "port", "extrapolated": False,
                "sample": (f"restated Prov_k(8) capture (naive Jacobi rounds, target-restricted) + exact "
                           f"compilation + FP64 gradient, single-threaded, {done} of {len(wl.qs)} queries in "
                           f"{secs:.1f} s")}
    pts, k = [], 0
    order = np.argsort(wl.nodes, kind="stable")
    t_tot = 0.0
    for i in order:
        n, s_, d_ = wl.instance(int(i))
        sess = O.Session(O.tc_program(s_, d_))
        counts, _, secs = sess.run(threads=1)
        sess.close()
        pts.append((max(len(s_), 1), counts["path"], secs))
        t_tot += secs
        k += 1
        if t_tot > budget_s or k >= 512:
            break
    big = sorted(pts)[len(pts) // 2:]  # fit on the larger half (the small ones are overhead-bound)
    a, b = _fit(big if len(big) >= 3 else pts)
    m_all = np.diff(wl.edge_off.astype(np.int64)).astype(np.float64)
    secs_all = float((a * np.maximum(m_all, 1.0) ** b).sum())
    return {"value": float(sum(p[1] for p in pts)) / t_tot, "unit": UNIT, "cores": 1, "kind": "port",
            "extrapolated": False,
            "sample": (f"restated reference interpreter, single-threaded, complete closures of the {k} smallest "
                       f"of {len(wl)} instances ({t_tot:.1f} s); per-instance fit t = a*E^b, b = {b:.2f}, "
                       f"summed over all instances: {secs_all:.3e} s (extrapolated)"),
            "exponent": b, "extrapolated_seconds": secs_all}


def fast_cpu(kind: str, wl, cores: int):
    """A fast all-core C++ baseline at the full size (not the reference's
    algorithm): Dijkstra per source (mssp), BFS per source (tc), sorted-list
    intersection per edge (tri), SCC condensation per instance (batch).
    Returns (baseline dict, the result it computed, for the parity check)."""
    import time as _t

    import oracle as O
    t0 = _t.perf_counter()
    if kind == "mssp":
        res = O.dijkstra_mssp(wl.sources, wl.src, wl.dst, wl.w, wl.source_w, threads=cores)
        what, tuples = "Dijkstra from each source (binary heap), sources across threads", res[0]
    elif kind == "tc":
        res = O.bfs_closure(wl.src, wl.dst, threads=cores)
        what, tuples = "BFS from every node, nodes across threads", res[0]
    elif kind == "tri":
        res = O.count_pattern(wl.src, wl.dst, threads=cores)
        what, tuples = "sorted-list intersection per edge (CSR), edges across threads", res
    elif kind == "batch":
        res = O.closure_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, threads=cores)
        what, tuples = ("closure count per instance by SCC condensation and bitset reachability, instances "
                        "across threads"), int(res[0].sum())
    else:
        return None, None
    secs = _t.perf_counter() - t0
    return ({"value": tuples / secs if secs > 0 else 0.0, "unit": UNIT, "cores": cores, "kind": "port",
             "seconds": secs, "sample": f"{what}; full workload, {tuples} tuples in {secs:.2f} s"}, res)


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    t0 = time.time()
    kind = args.workload
    if kind in INTERP_STEP:
        secs, tup, edges = [], 0, 0
        for _ in range(args.warmup + args.steps):
            edges, tup, s_ = _interp_point(kind, INTERP_STEP[kind])
            secs.append(s_)
        timed = secs[args.warmup:]
        value = tup * len(timed) / sum(timed) if sum(timed) > 0 else 0.0
        full_edges = {"mssp": 8 << args.scale, "tc": 50_000, "tri": 16 << args.scale}[kind]
        ext = interp_extrapolation(kind, full_edges, full_tuples=tup)  # only its fit is reported here
        sample = (f"one complete fixpoint per step of the restated reference interpreter (single-threaded "
                  f"nested-loop semi-naive, as strata run --semi-naive; the reference uses no threads) on a "
                  f"scaled-down instance of the same distribution ({_size_words(kind)} {INTERP_STEP[kind]}: "
                  f"{edges} edges, {tup} tuples)")
        cpu = {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample,
               "extrapolation": {"points": ext["points"], "exponent": ext["exponent"]}}
    else:
        wl = workload_for(0, args.scale, units_arg(args), kind)
        per = [interp_units(kind, wl, budget_s=10.0) for _ in range(args.warmup + args.steps)]
        value = float(np.mean([p["value"] for p in per[args.warmup:]]))
        cpu = {"value": value, "unit": unit_for(kind), "cores": 1, "kind": "port", "sample": per[-1]["sample"]}
        timed = [1000.0 / value if value else 0.0] * args.steps
    line = {
        "impl": "reference", "metric": metric_for(kind), "value": value, "unit": unit_for(kind),
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * sum(timed) / max(1, len(timed)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"mssp": "int64", "prov": "f64"}.get(kind, "u32"),
        "data": "synthetic", "config": config(args, world),
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": unit_for(kind), "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.time() - t0,
    }
    print(json.dumps(line), flush=True)
    if args.out:
        Path(args.out).write_text(json.dumps(line) + "\n")
    return 0


# ---------------------------------------------------------------- our arm
class Job:
    """One workload bound to an engine: its pinned host columns, the fixpoint
    call on resident device columns, and the host read-back of the result."""

    def __init__(self, kind, wl, eng, torch):
        self.kind, self.wl, self.eng, self.torch = kind, wl, eng, torch
        i32, i64 = np.int32, np.int64
        self.mode = 0
        if kind == "prov":
            cols = (("src", wl.src, i32), ("dst", wl.dst, i32), ("p64", wl.p64, np.float64),
                    ("p32", wl.p32, np.float32))
            self.host = {k: torch.from_numpy(np.ascontiguousarray(v).astype(dt)).pin_memory() for k, v, dt in cols}
            self.entry = "strata_prov_tc_capture + strata_circuits_compile/forward/grads"
            return
        if kind == "mssp":
            cols = (("sources", wl.sources, i32), ("sw", wl.source_w, i64), ("src", wl.src, i32),
                    ("dst", wl.dst, i32), ("w", wl.w, i64))
        else:
            cols = (("src", wl.src, i32), ("dst", wl.dst, i32))
            self.n_nodes = int(max(wl.src.max(), wl.dst.max())) + 1 if len(wl.src) else 1
        self.host = {k: torch.from_numpy(np.ascontiguousarray(v).astype(dt)).pin_memory() for k, v, dt in cols}
        self.entry = {"mssp": "strata_mssp_trop_dev", "tc": "strata_tc_bool_dev",
                      "tri": "strata_count_triangle_pattern_dev", "batch": "strata_tc_bool_batch_dev"}[kind]

    def run(self, d):
        """One fixpoint on device columns `d`: returns (result handle, tuples, stats)."""
        if self.kind == "mssp":
            rel = self.eng.mssp_dev(d["sources"], d["src"], d["dst"], d["w"], source_weights=d["sw"])
        elif self.kind == "tc" and getattr(self, "tc_shard", None):
            # path rows split across the ranks, Δ' slices all-gathered each round
            from strata_b200 import shard
            rank, world, dist = self.tc_shard
            part = self.eng.tc_shard(self.n_nodes, d["src"], d["dst"], rank, world)
            try:
                total, fp, rounds = shard.tc_bool_sharded([part], dist=dist, device="cuda")
                mine = part.summary()[0]
            finally:
                part.free()
            self.last = (total, fp, rounds)
            return None, mine, {"rounds": rounds, "fingerprint": fp, "path_total": total}
        elif self.kind == "tc":
            rel = self.eng.tc_bool_dev(d["src"], d["dst"])
        elif self.kind == "prov":
            self.eng.on_torch_stream()
            P, G, circ, info = self.eng.grad_queries(self.wl.n, d["src"], d["dst"], d["p64"], d["p32"],
                                                     self.wl.qs, self.wl.qt, k=8, chunks=4)
            self.torch.cuda.current_stream().synchronize()
            self.last = (P, G)
            nodes, levels = circ.shape()
            return circ, len(self.wl.qs), {"prov": info, "circuit_nodes": nodes, "circuit_levels": levels}
        elif self.kind == "batch":
            res = self.eng.tc_bool_batch(self.wl.nodes, self.wl.edge_off, d["src"], d["dst"], mode=self.mode)
            return None, int(res.counts.sum()), {"batch": res.stats}
        else:
            if getattr(self, "x_range", None):
                return None, self.eng.count_triangle_pattern_range_dev(d["src"], d["dst"], *self.x_range), None
            return None, self.eng.count_triangle_pattern_dev(d["src"], d["dst"]), None
        return rel, len(rel), rel.stats

    @staticmethod
    def free(handle):
        if handle is not None:
            handle.free()

    def out_buffers(self, n):
        torch = self.torch
        if self.kind in ("tri", "batch", "prov"):
            return None
        trop = self.kind == "mssp"
        return (torch.empty(n, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
                torch.empty(n, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
                torch.empty(n, dtype=torch.int64).pin_memory().numpy() if trop else None,
                torch.empty(n, dtype=torch.uint8).pin_memory().numpy() if trop else None)

    def fetch(self, handle, tuples, out):
        """Result to the host; returns the bytes read back."""
        if self.kind == "tri":
            return 8  # the u64 count, returned through the entry point's out-parameter
        if self.kind == "batch":
            return len(self.wl) * (8 + 8 + 4)  # per-instance count, fingerprint, rounds
        if self.kind == "tc" and getattr(self, "tc_shard", None):
            return 8 + 8 + 8  # |path|, fingerprint and rounds (a sharded closure stays on the ranks)
        if self.kind == "prov":
            P, G = self.last
            P.cpu()
            G.cpu()
            return P.numel() * P.element_size() + G.numel() * G.element_size()
        res = handle.to_host(out=out)
        assert len(res) == tuples
        return tuples * (4 + 4 + (8 + 1 if self.kind == "mssp" else 0))


def _timed_steps(step, free, stream, flush, steps, torch):
    """`steps` fixpoints, each bracketed by CUDA events on `stream`, with an
    L2 flush before each outside the interval.  Returns (ms, tuples, stats)."""
    total_ms, tuples, stats = 0.0, 0, None
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h, tuples, stats = step()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        free(h)
    return total_ms, tuples, stats


def _kernels(ks):
    return {k: {"launches": v[0], "ms": round(v[1], 3), "gbs": (v[2] / (v[1] / 1000.0) / 1e9) if v[1] else None}
            for k, v in ks.items() if v[0]}


def verify(kind: str, job, d, ref, eng, torch):
    """Check the engine's result on the timed workload against the CPU result
    `ref` (outside the timed region).  Returns a dict with "ok" and what was
    compared."""
    import oracle as O
    if kind in ("mssp", "tc"):
        h, n, _ = job.run(d)
        try:
            fp = h.fingerprint()
        finally:
            h.free()
        return {"ok": bool(n == ref[0] and fp == ref[1]), "tuples": int(n),
                "what": "count and order-independent fingerprint of every tuple (and weight) vs the CPU baseline"}
    if kind == "tri":
        _, n, _ = job.run(d)
        return {"ok": bool(n == ref), "what": "exact triangle count vs the CPU baseline", "count": int(n)}
    if kind == "batch":
        res = eng.tc_bool_batch(job.wl.nodes, job.wl.edge_off, d["src"], d["dst"], mode=0)
        ok = bool(np.array_equal(res.counts, ref[0]) and np.array_equal(res.fps, ref[1]))
        return {"ok": ok, "what": "every instance's |path| and fingerprint vs SCC-condensation closures"}
    if kind == "prov":
        wl = job.wl
        P, G = (t.cpu().numpy() for t in job.last)
        proofs = eng.prov_capture(wl.n, d["src"], d["dst"], d["p64"], wl.qs, wl.qt, k=8)
        worst_p, worst_g, leaves = 0.0, 0.0, 0
        for q in range(len(wl.qs)):
            want_p, want_g, _ = O.compile_grad(proofs.query(q), wl.p64)
            if want_p == 0.0:
                worst_p = max(worst_p, abs(float(P[q])))
                continue
            worst_p = max(worst_p, abs(float(P[q]) - want_p) / want_p)
            nz = want_g != 0.0
            leaves += int(nz.sum())
            if nz.any():
                worst_g = max(worst_g, float((np.abs(G[q][nz] - want_g[nz]) / np.abs(want_g[nz])).max()))
            if (G[q][~nz] != 0.0).any():
                worst_g = float("inf")
        return {"ok": bool(worst_p <= 1e-5 and worst_g <= 1e-5), "p_max_rel_err": worst_p,
                "grad_max_rel_err": worst_g, "grad_entries": leaves,
                "what": ("P (FP32) and every nonzero gradient entry of every query vs the FP64 circuit oracle "
                         "(exact compilation of the same proof sets, f64 WMC and adjoint)")}
    return None


def run_ours(args):
    import torch

    import strata_b200 as S

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    sharded = bool(args.shard and world > 1 and args.workload in ("mssp", "tc", "batch", "prov", "tri"))
    wl = workload_for(0 if sharded else rank, args.scale, units_arg(args), args.workload)
    x_range = None
    if sharded:
        from strata_b200 import shard
        if args.workload == "mssp":
            mine, idx = shard.shard_sources(wl.sources, rank, world)
            wl.sources, wl.source_w = mine, wl.source_w[idx]
        elif args.workload == "batch":
            wl = shard.batch_subset(wl, shard.shard_instances(wl.nodes, rank, world))
        elif args.workload == "tri":
            x_range = shard.shard_vertices(int(max(wl.src.max(), wl.dst.max())) + 1, rank, world)
        elif args.workload == "tc":
            pass  # the Job splits the path rows; the edge list is replicated
        else:
            qi = shard.shard_queries(wl.qt, rank, world)
            wl.qs, wl.qt = wl.qs[qi], wl.qt[qi]
    eng = S.Engine(local, tuned=args.tuned)
    eng.set_plan(PLANS[args.plan])
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    job = Job(args.workload, wl, eng, torch)
    job.x_range = x_range
    if sharded and args.workload == "tc":
        job.tc_shard = (rank, world, pg)
        job.entry = "strata_tc_shard_create/seed/round/summary + NCCL all-gather of the Δ' rows"
    with torch.cuda.stream(stream):
        d = {k: v.to("cuda", non_blocking=True) for k, v in job.host.items()}
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    stream.synchronize()

    def step():
        with torch.cuda.stream(stream):
            return job.run(d)

    for _ in range(args.warmup):
        job.free(step()[0])
    # ---- timed region: device-only fixpoints (inputs resident in HBM)
    eng.set_profiling(True)
    eng.reset_kernel_stats()
    clocks = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = eng.launches()
    total_ms, tuples, stats = _timed_steps(step, job.free, stream, flush, args.steps, torch)
    torch.cuda.synchronize()
    launches = eng.launches() - launches0
    clk = clocks.stop()
    kstats = eng.kernel_stats()
    eng.set_profiling(False)

    # ---- the sort-merge plan on the same inputs (reported beside the headline)
    sort_plan = None
    if not args.no_sort_plan and args.workload in ("mssp", "tc") and args.plan == "auto" and not sharded:
        eng.set_plan(PLANS["sort-merge"])
        job.free(step()[0])  # warm its buffers
        eng.set_profiling(True)
        eng.reset_kernel_stats()
        sp_ms, sp_tuples, sp_stats = _timed_steps(step, job.free, stream, flush, args.steps, torch)
        assert sp_tuples == tuples
        sk = eng.kernel_stats()
        eng.set_profiling(False)
        eng.set_plan(PLANS["auto"])
        sort_plan = {"plan": "sort-merge (radix sort + run reduction + merge-path diff per round)",
                     "ms_per_step": sp_ms / args.steps, "value": tuples * args.steps / (sp_ms / 1000.0),
                     "phase_ms": {k: round(sp_stats[k + "_ms"], 3)
                                  for k in ("setup", "join", "sort", "diff", "merge", "finish")},
                     "kernels": _kernels(sk)}
    # ---- the same fixpoint in int64 weight lanes (what weights beyond the
    # int32 proof bound run in), reported beside the headline
    wide = None
    if args.workload == "mssp" and args.plan == "auto" and not sharded:
        eng.set_knob(9, 8)
        job.free(step()[0])  # warm its buffers
        eng.set_profiling(True)
        eng.reset_kernel_stats()
        wd_ms, wd_tuples, wd_stats = _timed_steps(step, job.free, stream, flush, args.steps, torch)
        assert wd_tuples == tuples
        wk = eng.kernel_stats()
        eng.set_profiling(False)
        eng.set_knob(9, 0)
        wide = {"lanes": "int64 weight lanes forced (STRATA_KNOB_WEIGHT_LANES = 8), same plan selection",
                "plan": {1: "sort-merge", 2: "direct-addressed"}.get(wd_stats["plan"], "?"),
                "weight_bytes": wd_stats["weight_bytes"], "ms_per_step": wd_ms / args.steps,
                "value": tuples * args.steps / (wd_ms / 1000.0), "kernels": _kernels(wk)}
    # ---- batched form: the same instances one per launch (host-driven rounds)
    per_launch = None
    if args.workload == "batch":
        job.mode = 1
        eng.set_profiling(False)
        pl_ms, pl_tuples, pl_stats = _timed_steps(step, job.free, stream, flush, 1, torch)
        job.mode = 0
        assert pl_tuples == tuples
        per_launch = {"mode": "one instance per launch, same kernels, host-driven rounds (1 step)",
                      "ms_per_step": pl_ms, "value": pl_tuples / (pl_ms / 1000.0),
                      "speedup_of_batched": pl_ms / (total_ms / args.steps),
                      "round_launches": pl_stats["batch"]["round_launches"]}
        # the same comparison on the instances with n <= 5,000 (three quarters
        # of them, a sliver of the work): where launches and host round trips,
        # not the rows' bytes, set the time
        from strata_b200 import shard
        small = np.flatnonzero(np.asarray(job.wl.nodes) <= 5000)
        sub = shard.batch_subset(job.wl, small)
        ds, dd = (torch.from_numpy(np.ascontiguousarray(a).astype(np.int32)).cuda() for a in (sub.src, sub.dst))
        torch.cuda.synchronize()
        times = {}
        for mode in (0, 1, 0, 1):
            with torch.cuda.stream(stream):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                eng.tc_bool_batch(sub.nodes, sub.edge_off, ds, dd, mode=mode)
                e1.record(stream)
            e1.synchronize()
            times[mode] = e0.elapsed_time(e1)  # the second run of each mode (warm)
        per_launch["small_instances"] = {"instances": int(len(small)), "n_max": 5000,
                                         "batched_ms": times[0], "one_per_launch_ms": times[1],
                                         "speedup_of_batched": times[1] / times[0]}
    if pg:
        t = torch.tensor([total_ms, float(tuples)], dtype=torch.float64, device="cuda")
        mx = t.clone()
        pg.all_reduce(mx, op=pg.ReduceOp.MAX)
        sm = t.clone()
        pg.all_reduce(sm, op=pg.ReduceOp.SUM)
        max_ms, all_tuples = float(mx[0]), float(sm[1])
    else:
        max_ms, all_tuples = total_ms, float(tuples)
    ms_per_step = max_ms / args.steps
    value = all_tuples * args.steps / (max_ms / 1000.0)

    # ---- e2e: pinned host inputs -> device -> fixpoint -> result on the host
    e2e = None
    if not args.no_e2e:
        out_host = job.out_buffers(tuples)
        h2d = sum(v.numel() * v.element_size() for v in job.host.values())
        e2e_ms, d2h = 0.0, 0
        for i in range(args.steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            with torch.cuda.stream(stream):
                dd = {k: v.to("cuda", non_blocking=True) for k, v in job.host.items()}
            h, n_out, _ = job.run(dd)
            d2h = job.fetch(h, n_out, out_host)
            t1 = time.perf_counter()
            assert n_out == tuples
            job.free(h)
            del dd
            if i > 0:  # first iteration is a warm-up
                e2e_ms += 1000 * (t1 - t0)
        e2e_val = tuples * args.steps / (e2e_ms / 1000.0)
        if pg:
            t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            e2e_val = all_tuples * args.steps / (float(t[0]) / 1000.0)
        e2e = {"value": e2e_val, "unit": unit_for(args.workload), "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "path": f"pinned host columns -> torch H2D -> {job.entry}"
                       + (" (count out-parameter)" if args.workload == "tri" else
                          " (count, fingerprint, rounds)" if getattr(job, "tc_shard", None) else
                          " -> strata_rel_to_host (pinned)")}

    # ---- roofline of the dominant kernel
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom = max(kstats.items(), key=lambda kv: kv[1][1])
    name, (kl, kms, kbytes) = dom
    achieved = (kbytes / kl) / ((kms / kl) / 1000.0) / 1e9 if kl and kms else 0.0
    roof = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "peak_source": peak_src,
            "unit": "GB/s", "frac": achieved / peak if peak else None,
            "traffic": TRAFFIC.get((args.workload, name)), "launches_per_step": kl / args.steps,
            "avg_launch_us": 1000 * kms / kl if kl else None,
            "algorithmic_bytes_per_launch": kbytes / kl if kl else None,
            "kernels": _kernels(kstats)}

    cpu, cpu_fast, check = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        if args.workload in INTERP_SIZES:
            cpu = interp_extrapolation(args.workload, len(wl.src), int(all_tuples))
        else:
            cpu = interp_units(args.workload, wl)
        cpu_fast, ref_result = fast_cpu(args.workload, wl, cores)
        if args.workload == "prov" or ref_result is not None:
            with torch.cuda.stream(stream):
                check = verify(args.workload, job, d, ref_result, eng, torch)
            torch.cuda.synchronize()

    if rank == 0:
        wb = stats.get("weight_bytes", 0) if stats else 0
        line = {
            "metric": metric_for(args.workload), "value": value, "unit": unit_for(args.workload), "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": {4: "int32", 8: "int64"}.get(wb, "u32"),
            "data": "synthetic", "config": config(args, world),
            "tuples_per_step": int(all_tuples),
            "clocks": clk, "e2e": e2e, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
            "cpu_fast": cpu_fast, "check": check,
        }
        if stats and "prov" in stats:
            line.update({"dtype": "f32 (circuits), f64 (proof weights, root sums, leaf gradients)",
                         "prov": {**stats["prov"], "circuit_nodes": stats["circuit_nodes"],
                                  "circuit_levels": stats["circuit_levels"]}})
        elif stats and "batch" in stats:
            b = stats["batch"]
            line.update({"dtype": "u32", "plan": "bit rows, batched waves",
                         "batch": {k: b[k] for k in ("instances", "waves", "graph_launches", "round_launches",
                                                     "rounds_max", "round_bytes")},
                         "one_per_launch": per_launch})
        elif stats:
            line.update({
                "plan": {1: "sort-merge", 2: "direct-addressed", 3: "bit rows"}.get(stats["plan"], "?"),
                "rounds": stats["rounds"], "candidates_per_step": stats["candidates"],
                "key_bits": stats["key_bits"], "weight_bytes": stats["weight_bytes"],
                "phase_ms": {k: round(stats[k + "_ms"], 3)
                             for k in ("setup", "join", "sort", "diff", "merge", "finish")},
                "sort_merge_plan": sort_plan, "wide_lanes": wide})
        print(json.dumps(line), flush=True)
        if args.out:
            Path(args.out).write_text(json.dumps(line) + "\n")
    eng.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
