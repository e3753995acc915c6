"""Autotuner for the engine's kernel knobs.

Sweeps each knob of `strata_ctx_set_knob` over its choices on synthetic
inputs of a representative size, times every choice with CUDA events on the
engine's stream, and keeps the fastest.  The result is cached as JSON (per
GPU name) and applied by :func:`apply_cached` — `Engine(..., tuned=True)`
does that on creation.  Knobs change speed only; results are identical for
every choice (the parity tests compare every choice against the default).

    python -m strata_b200.tune          # sweep, print, write the cache
"""
from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path

KNOBS = {
    # radix tile keys per thread — knob id: (key bytes, choices, significant key bits of the probe)
    1: (4, (11, 15, 19, 23), 26),
    2: (8, (7, 9, 13), 40),
}
# other knobs: id -> choices (0 = the built-in default)
OTHER = {
    3: (1, 2, 3),             # triangle membership test: hash set / binary search / bitmap filter
    4: (2, 4, 8, 16, 32),     # bit-row rounds per CUDA-graph replay (batched closure)
    5: (0, 2, 4, 8),          # resident round-kernel blocks per SM (0 = occupancy limit)
    7: (1, 2, 3),             # radix digit ranking: ballots / match instruction / shared masks
    8: (8, 12, 16, 20, 24, 33),  # Δ-word members from which the bit-lane expand path runs (33 = never)
}


def cache_path() -> Path:
    p = os.environ.get("STRATA_B200_TUNE_CACHE")
    if p:
        return Path(p)
    return Path.home() / ".cache" / "strata_b200" / "tune.json"


def _gpu_name() -> str:
    import torch
    return torch.cuda.get_device_name(0)


def _time_sort(eng, torch, n: int, key_bytes: int, bits: int, reps: int = 5) -> float:
    kdt = torch.int32 if key_bytes == 4 else torch.int64
    keys = torch.randint(0, 1 << bits, (n,), dtype=torch.int64, device="cuda").to(kdt)
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ko, vo = torch.empty_like(keys), torch.empty_like(vals)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)

    def run():
        eng._check(eng.lib.strata_op_sort(eng.ctx, key_bytes, 4, C.c_void_p(keys.data_ptr()),
                                          C.c_void_p(vals.data_ptr()), C.c_void_p(ko.data_ptr()),
                                          C.c_void_p(vo.data_ptr()), n, bits))

    run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    e1.synchronize()
    eng.set_stream(None)
    return e0.elapsed_time(e1) / reps


def _time_call(torch, fn, reps: int = 3) -> float:
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def sweep(n: int = 64_000_000, verbose: bool = True, batch_instances: int = 512) -> dict:
    """Time every choice of every knob; return {knob: best value} plus timings."""
    import numpy as np
    import torch

    from . import gen
    from .gpu import Engine
    eng = Engine(0)
    best, timings = {}, {}

    def record(knob, res):
        best[knob] = min(res, key=res.get)
        timings[knob] = res
        if verbose:
            for v, t in res.items():
                print(f"knob {knob} = {v}: {t:.3f} ms")

    try:
        for knob, (kb, choices, bits) in KNOBS.items():
            res = {}
            for v in choices:
                eng.set_knob(knob, v)
                res[v] = _time_sort(eng, torch, n if kb == 4 else n // 2, kb, bits)
            eng.set_knob(knob, 0)
            record(knob, res)
        # radix ranking method (u32 keys at the tuned tile size)
        res = {}
        eng.set_knob(1, best[1])
        for v in OTHER[7]:
            eng.set_knob(7, v)
            res[v] = _time_sort(eng, torch, n, 4, 26)
        eng.set_knob(7, 0)
        eng.set_knob(1, 0)
        record(7, res)
        # triangle probe on an oriented R-MAT graph
        tw = gen.triangle_workload(scale=18, seed=7)
        tx = torch.from_numpy(tw.src.astype(np.int32)).cuda()
        ty = torch.from_numpy(tw.dst.astype(np.int32)).cuda()
        res = {}
        for v in OTHER[3]:
            eng.set_knob(3, v)
            res[v] = _time_call(torch, lambda: eng.count_triangle_pattern_dev(tx, ty))
        eng.set_knob(3, 0)
        record(3, res)
        # batched closure knobs on a mixed-size batch
        bw = gen.batch_tc_workload(n_inst=batch_instances, n_min=100, n_max=20_000, seed=9)
        bs = torch.from_numpy(bw.src.astype(np.int32)).cuda()
        bd = torch.from_numpy(bw.dst.astype(np.int32)).cuda()
        for knob in (4, 5):
            res = {}
            for v in OTHER[knob]:
                eng.set_knob(knob, v)
                res[v] = _time_call(torch, lambda: eng.tc_bool_batch(bw.nodes, bw.edge_off, bs, bd, mode=0), reps=2)
            eng.set_knob(knob, 0)
            record(knob, res)
        # direct-addressed Trop rounds: multi-source shortest paths on R-MAT-18
        mw = gen.mssp_workload(scale=18, n_sources=64, seed=11)
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).astype(dt)).cuda()
        ms = (t(mw.sources, np.int32), t(mw.src, np.int32), t(mw.dst, np.int32), t(mw.w, np.int64),
              t(mw.source_w, np.int64))
        res = {}
        for v in OTHER[8]:
            eng.set_knob(8, v)
            res[v] = _time_call(torch, lambda: eng.mssp_dev(*ms[:4], source_weights=ms[4]).free())
        eng.set_knob(8, 0)
        record(8, res)
    finally:
        eng.close()
    return {"gpu": _gpu_name(), "best": best, "timings_ms": timings, "n": n}


def save(result: dict, path: Path | None = None) -> Path:
    path = path or cache_path()
    path.parent.mkdir(parents=True, exist_ok=True)
    data = {}
    if path.exists():
        try:
            data = json.loads(path.read_text())
        except ValueError:
            data = {}
    data[result["gpu"]] = {str(k): v for k, v in result["best"].items()}
    path.write_text(json.dumps(data, indent=1))
    return path


def load(path: Path | None = None, gpu: str | None = None) -> dict:
    """Cached {knob: value} for `gpu` (default: this process's device 0)."""
    path = path or cache_path()
    if not path.exists():
        return {}
    try:
        data = json.loads(path.read_text())
    except ValueError:
        return {}
    entry = data.get(gpu if gpu is not None else _gpu_name(), {})
    out = {}
    for k, v in entry.items():
        k, v = int(k), int(v)
        if (k in KNOBS and v in KNOBS[k][1]) or (k in OTHER and v in OTHER[k]):
            out[k] = v
    return out


def apply_cached(eng, path: Path | None = None) -> dict:
    """Set the cached knob values of this GPU on `eng` (no-op without a cache)."""
    vals = load(path)
    for k, v in vals.items():
        eng.set_knob(k, v)
    return vals


if __name__ == "__main__":
    r = sweep()
    print(json.dumps(r))
    print("cache:", save(r))
