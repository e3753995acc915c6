"""The engine's public API, mirroring the reference GPU crate.

Function names, argument meaning and error behaviour follow
``strata-gpu/src/lib.rs:67-147``:

* ``transitive_closure_bool(edges)``        (lib.rs:67, tc.rs:31)
* ``shortest_paths_trop(edges)``            (lib.rs:84, trop.rs:51)
* ``count_triangles(edges)``                (lib.rs:99, wcoj.rs:136)
* ``count_4cliques(edges)``                 (lib.rs:114, wcoj.rs:166)
* ``intern_terms(keys)``                    (lib.rs:133, sort.rs:206)
* ``binary_plan_intermediate(edges)``       (lib.rs:140, wcoj.rs:190)

plus the multi-source Trop fixpoint of the benchmark program
(``mssp_trop``) and the count aggregate over a directed relation
(``count_triangle_pattern``).  Inputs need not be sorted or deduplicated;
outputs are sorted by ``(src, dst)``.  Errors raise :class:`GpuError`
subclasses; a negative-weight cycle is :class:`NegativeWeightCycle` (the
reference reports it as ``GpuError::Cuda("negative-weight cycle…")``,
trop.rs:87-89) and a Trop overflow is :class:`TropOverflow` (the
interpreter's ``EvalError::Overflow``, strata-eval/src/naive.rs:31).

Every call runs on the GPU through ``libstrata_b200.so``; nothing here
computes a result on the CPU.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

POS_INF = float("inf")  # how +inf is shown in Python-level tuples


class GpuError(Exception):
    """Error from the GPU engine (mirror of ``GpuError``, strata-gpu/src/lib.rs:14)."""

    code = L.E_CUDA


class NotBuilt(GpuError):
    """No CUDA device / library (``GpuError::NotBuilt``)."""

    code = L.E_NOT_BUILT


class Cuda(GpuError):
    """A CUDA runtime failure (``GpuError::Cuda``)."""

    code = L.E_CUDA


class InvalidArgument(GpuError):
    code = L.E_INVALID


class OutOfMemory(GpuError):
    code = L.E_OOM


class TropOverflow(GpuError):
    """Finite Trop ⊗ overflowed i64 (``EvalError::Overflow``)."""

    code = L.E_OVERFLOW


class NegativeWeightCycle(GpuError):
    """Trop stratum exceeded the Bellman-Ford cap (``EvalError::NegativeWeightCycle``)."""

    code = L.E_NEG_CYCLE


class Timeout(GpuError):
    code = L.E_TIMEOUT


class Unsupported(GpuError):
    code = L.E_UNSUPPORTED


class WeightRange(GpuError):
    """Finite weights spanning nearly all of i64: no 64-bit code keeps them apart from +inf."""

    code = L.E_WEIGHT_RANGE


_ERRORS = {c.code: c for c in (NotBuilt, Cuda, InvalidArgument, OutOfMemory, TropOverflow,
                               NegativeWeightCycle, Timeout, Unsupported, WeightRange)}


def _raise(code: int, msg: str):
    raise _ERRORS.get(code, GpuError)(f"{L.STATUS_NAMES.get(code, code)}: {msg}")


@dataclass
class TropRelation:
    """A Trop relation: columns ``src, dst, w`` and ``inf`` (1 where w = +inf)."""

    src: np.ndarray
    dst: np.ndarray
    w: np.ndarray
    inf: np.ndarray
    stats: dict = field(default_factory=dict)

    def __len__(self) -> int:
        return len(self.src)

    def tuples(self) -> list[tuple[int, int, float | int]]:
        return [(int(s), int(d), POS_INF if i else int(w))
                for s, d, w, i in zip(self.src, self.dst, self.w, self.inf)]


@dataclass
class BoolRelation:
    """A Bool relation: columns ``src, dst``."""

    src: np.ndarray
    dst: np.ndarray
    stats: dict = field(default_factory=dict)

    def __len__(self) -> int:
        return len(self.src)

    def tuples(self) -> list[tuple[int, int]]:
        return list(zip(self.src.tolist(), self.dst.tolist()))


def _u32(a) -> np.ndarray:
    a = np.asarray(a)
    if a.size and (a.min() < 0 or a.max() > 0xFFFFFFFF):
        raise InvalidArgument("ids must fit in u32")
    return np.ascontiguousarray(a, dtype=np.uint32)


def _split_pairs(edges) -> tuple[np.ndarray, np.ndarray]:
    if isinstance(edges, tuple) and len(edges) == 2 and not np.isscalar(edges[0]):
        return _u32(edges[0]), _u32(edges[1])
    a = np.asarray(list(edges) if not isinstance(edges, np.ndarray) else edges)
    if a.size == 0:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    a = a.reshape(-1, 2)
    return _u32(a[:, 0]), _u32(a[:, 1])


def _split_weighted(edges) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(src, dst, w) triples; w may be POS_INF.  Or a tuple of 3/4 columns."""
    if isinstance(edges, tuple) and len(edges) in (3, 4) and not np.isscalar(edges[0]):
        s, d, w = _u32(edges[0]), _u32(edges[1]), np.ascontiguousarray(edges[2], dtype=np.int64)
        inf = (np.ascontiguousarray(edges[3], dtype=np.uint8) if len(edges) == 4
               else np.zeros(len(s), np.uint8))
        return s, d, w, inf
    rows = list(edges)
    if not rows:
        z = np.zeros(0, np.uint32)
        return z, z, np.zeros(0, np.int64), np.zeros(0, np.uint8)
    s = _u32([r[0] for r in rows])
    d = _u32([r[1] for r in rows])
    inf = np.array([1 if r[2] == POS_INF else 0 for r in rows], dtype=np.uint8)
    w = np.array([0 if r[2] == POS_INF else int(r[2]) for r in rows], dtype=np.int64)
    return s, d, w, inf


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class Engine:
    """A context on one CUDA device (its own stream, byte cap, status word).

    Not thread-safe; create one Engine per thread.  ``mem_cap`` bounds the
    device bytes the engine may hold (0 = unbounded).
    """

    def __init__(self, device: int = 0, mem_cap: int = 0, profiling: bool = False, tuned: bool = False):
        self.lib = L.load()
        ctx = L.ctxp()
        rc = self.lib.strata_ctx_create(device, mem_cap, C.byref(ctx))
        if rc != L.OK:
            _raise(rc, "cannot create a context on CUDA device %d" % device)
        self.ctx = ctx
        self.device = device
        if profiling:
            self.lib.strata_ctx_set_profiling(self.ctx, 1)
        if tuned:  # knob values cached by `python -m strata_b200.tune` for this GPU
            from . import tune
            tune.apply_cached(self)

    # -- plumbing ---------------------------------------------------------
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.strata_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != L.OK:
            _raise(rc, self.lib.strata_last_error(self.ctx).decode(errors="replace"))

    def set_stream(self, stream_handle: int | None):
        """Run on an existing ``cudaStream_t`` (e.g. ``torch.cuda.Stream().cuda_stream``)."""
        self._check(self.lib.strata_ctx_set_stream(self.ctx, C.c_void_p(stream_handle or 0)))
        self._stream = stream_handle or 0

    def synchronize(self):
        """Wait for the work queued on the context's stream."""
        self._check(self.lib.strata_ctx_synchronize(self.ctx))

    def on_torch_stream(self) -> bool:
        """Order the context's next asynchronous calls (the circuit kernels)
        with torch's current CUDA stream: run on that stream when it is a
        created stream; for the legacy default stream (handle 0, which a
        non-blocking stream does not wait for) finish torch's queued work now
        and return True — the caller then synchronizes after its call."""
        import torch
        h = torch.cuda.current_stream().cuda_stream
        if h:
            if getattr(self, "_stream", None) != h:
                self.set_stream(h)
            return False
        torch.cuda.current_stream().synchronize()
        if getattr(self, "_stream", None):
            self.set_stream(None)
        return True

    def set_plan(self, plan: int):
        """0 automatic, 1 sort-merge, 2 direct-addressed, 3 bit rows (Bool closure only);
        results are identical."""
        self._check(self.lib.strata_ctx_set_plan(self.ctx, plan))

    def set_knob(self, knob: int, value: int):
        """Tuning knob (1: radix keys/thread for u32 keys, 2: for u64 keys, 3: triangle
        probe 1 hash / 2 binary search; 0 = default).  Results never depend on knobs."""
        self._check(self.lib.strata_ctx_set_knob(self.ctx, knob, value))

    def set_profiling(self, on: bool):
        self._check(self.lib.strata_ctx_set_profiling(self.ctx, 1 if on else 0))

    def launches(self) -> int:
        return int(self.lib.strata_ctx_launches(self.ctx))

    def kernel_stats(self) -> dict:
        """{kernel name: (launches, summed ms, algorithmic bytes)} while profiling."""
        out = {}
        for kid, name in L.KERNELS.items():
            n, ms, b = C.c_uint64(), C.c_double(), C.c_uint64()
            self._check(self.lib.strata_ctx_kernel_stats(self.ctx, kid, C.byref(n), C.byref(ms), C.byref(b)))
            out[name] = (int(n.value), float(ms.value), int(b.value))
        return out

    def reset_kernel_stats(self):
        self._check(self.lib.strata_ctx_reset_kernel_stats(self.ctx))

    def mem(self) -> tuple[int, int]:
        a, b = C.c_uint64(), C.c_uint64()
        self._check(self.lib.strata_ctx_mem(self.ctx, C.byref(a), C.byref(b)))
        return a.value, b.value

    def _take(self, p, n, dtype) -> np.ndarray:
        """Copy a library-malloc'd buffer into numpy and free it."""
        out = np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0, dtype)
        self.lib.strata_free(C.cast(p, C.c_void_p))
        return out.astype(dtype, copy=False)

    # -- whole fixpoints (host buffers) ------------------------------------
    def transitive_closure_bool(self, edges) -> BoolRelation:
        s, d = _split_pairs(edges)
        os_, od = L.u32p(), L.u32p()
        n = C.c_uint64()
        st = L.FixStats()
        self._check(self.lib.strata_transitive_closure_bool(
            self.ctx, _ptr(s, C.c_uint32), _ptr(d, C.c_uint32), len(s), C.byref(os_), C.byref(od),
            C.byref(n), C.byref(st)))
        return BoolRelation(self._take(os_, n.value, np.uint32), self._take(od, n.value, np.uint32),
                            st.as_dict())

    def shortest_paths_trop(self, edges) -> TropRelation:
        s, d, w, inf = _split_weighted(edges)
        os_, od, ow, oi = L.u32p(), L.u32p(), L.i64p(), L.u8p()
        n = C.c_uint64()
        st = L.FixStats()
        self._check(self.lib.strata_shortest_paths_trop(
            self.ctx, _ptr(s, C.c_uint32), _ptr(d, C.c_uint32), _ptr(w, C.c_int64),
            _ptr(inf, C.c_uint8), len(s), C.byref(os_), C.byref(od), C.byref(ow), C.byref(oi),
            C.byref(n), C.byref(st)))
        m = n.value
        return TropRelation(self._take(os_, m, np.uint32), self._take(od, m, np.uint32),
                            self._take(ow, m, np.int64), self._take(oi, m, np.uint8), st.as_dict())

    def mssp_trop(self, sources, edges, source_weights=None, source_inf=None) -> TropRelation:
        """dist(S,Y) :- src(S), edge(S,Y).  dist(S,Z) :- dist(S,Y), edge(Y,Z)."""
        src = _u32(sources)
        sw = None if source_weights is None else np.ascontiguousarray(source_weights, dtype=np.int64)
        si = None if source_inf is None else np.ascontiguousarray(source_inf, dtype=np.uint8)
        s, d, w, inf = _split_weighted(edges)
        os_, od, ow, oi = L.u32p(), L.u32p(), L.i64p(), L.u8p()
        n = C.c_uint64()
        st = L.FixStats()
        self._check(self.lib.strata_mssp_trop(
            self.ctx, _ptr(src, C.c_uint32), None if sw is None else _ptr(sw, C.c_int64),
            None if si is None else _ptr(si, C.c_uint8), len(src),
            _ptr(s, C.c_uint32), _ptr(d, C.c_uint32), _ptr(w, C.c_int64), _ptr(inf, C.c_uint8),
            len(s), C.byref(os_), C.byref(od), C.byref(ow), C.byref(oi), C.byref(n), C.byref(st)))
        m = n.value
        return TropRelation(self._take(os_, m, np.uint32), self._take(od, m, np.uint32),
                            self._take(ow, m, np.int64), self._take(oi, m, np.uint8), st.as_dict())

    def _count(self, fn, edges) -> int:
        a, b = _split_pairs(edges)
        out = C.c_uint64()
        self._check(fn(self.ctx, _ptr(a, C.c_uint32), _ptr(b, C.c_uint32), len(a), C.byref(out)))
        return int(out.value)

    def count_triangles(self, edges) -> int:
        return self._count(self.lib.strata_count_triangles, edges)

    def count_4cliques(self, edges) -> int:
        return self._count(self.lib.strata_count_4cliques, edges)

    def count_triangle_pattern(self, edges) -> int:
        return self._count(self.lib.strata_count_triangle_pattern, edges)

    def binary_plan_intermediate(self, edges) -> int:
        return self._count(self.lib.strata_binary_plan_intermediate, edges)

    def intern_terms(self, keys) -> np.ndarray:
        k = np.ascontiguousarray(keys, dtype=np.uint64)
        ids = np.zeros(len(k), np.uint32)
        nd = C.c_uint64()
        self._check(self.lib.strata_intern_terms(self.ctx, _ptr(k, C.c_uint64), len(k),
                                                 _ptr(ids, C.c_uint32), C.byref(nd)))
        return ids

    # -- device-resident fixpoints (torch tensors or raw device pointers) ----
    def tc_bool_dev(self, src, dst, n=None) -> "DeviceRelation":
        n = _len(src) if n is None else n
        rel = L.relp()
        st = L.FixStats()
        self._check(self.lib.strata_tc_bool_dev(self.ctx, _dp(src), _dp(dst), n, C.byref(rel), C.byref(st)))
        return DeviceRelation(self, rel, st.as_dict())

    def trop_paths_dev(self, src, dst, w, inf=None, n=None) -> "DeviceRelation":
        n = _len(src) if n is None else n
        rel = L.relp()
        st = L.FixStats()
        self._check(self.lib.strata_trop_paths_dev(self.ctx, _dp(src), _dp(dst), _dp(w), _dp(inf), n,
                                                   C.byref(rel), C.byref(st)))
        return DeviceRelation(self, rel, st.as_dict())

    def mssp_dev(self, sources, esrc, edst, ew, source_weights=None, source_inf=None, einf=None,
                 n_sources=None, n_edges=None) -> "DeviceRelation":
        ns = _len(sources) if n_sources is None else n_sources
        ne = _len(esrc) if n_edges is None else n_edges
        rel = L.relp()
        st = L.FixStats()
        self._check(self.lib.strata_mssp_trop_dev(
            self.ctx, _dp(sources), _dp(source_weights), _dp(source_inf), ns, _dp(esrc), _dp(edst),
            _dp(ew), _dp(einf), ne, C.byref(rel), C.byref(st)))
        return DeviceRelation(self, rel, st.as_dict())

    # -- sharded Bool closure (one rank's share) --------------------------
    def tc_shard(self, n_nodes: int, src, dst, rank: int, world: int) -> "TcShard":
        """Rank `rank`'s share of a Bool closure split by path rows over
        `world` ranks (`strata_b200.shard.tc_bool_sharded` runs the rounds).
        ``src``/``dst`` are device tensors (int32 or uint32 ids)."""
        if not (hasattr(src, "data_ptr") and hasattr(dst, "data_ptr")):
            raise InvalidArgument("tc_shard takes device tensors")
        if _len(src) != _len(dst):
            raise InvalidArgument("src and dst must have the same length")
        _torch_sync(src)
        out = C.c_void_p()
        self._check(self.lib.strata_tc_shard_create(self.ctx, n_nodes, _dp(src), _dp(dst), _len(src), rank, world,
                                                     C.byref(out)))
        return TcShard(self, out, rank, world, keep=(src, dst))

    # -- batched Bool reachability ---------------------------------------
    def tc_bool_batch(self, nodes, edge_off, src, dst, mode: int = 0) -> "BatchResult":
        """Closures of many independent graphs (instance i: nodes [0, nodes[i]),
        edges src/dst[edge_off[i]:edge_off[i+1]]), summarised per instance by
        |path|, Σ mix64(X)·c^Z and the round count.  ``src``/``dst`` may be
        host arrays or device tensors.  mode 0 batched (graph-replayed
        persistent rounds), 1 one instance per launch."""
        nd = np.ascontiguousarray(nodes, dtype=np.uint32)
        eo = np.ascontiguousarray(edge_off, dtype=np.uint64)
        n_inst = len(nd)
        if len(eo) != n_inst + 1:
            raise InvalidArgument("edge_off needs one more entry than nodes")
        m = int(eo[-1]) if n_inst else 0
        if _len(src) != m or _len(dst) != m:
            raise InvalidArgument("src and dst must hold edge_off[-1] edges")
        counts = np.zeros(n_inst, np.uint64)
        fps = np.zeros(n_inst, np.uint64)
        rounds = np.zeros(n_inst, np.uint32)
        st = L.BatchStats()
        if hasattr(src, "data_ptr"):
            self._check(self.lib.strata_tc_bool_batch_dev(
                self.ctx, n_inst, _ptr(nd, C.c_uint32), _ptr(eo, C.c_uint64), _dp(src), _dp(dst), mode,
                _ptr(counts, C.c_uint64), _ptr(fps, C.c_uint64), _ptr(rounds, C.c_uint32), C.byref(st)))
        else:
            s_, d_ = _u32(src), _u32(dst)
            self._check(self.lib.strata_tc_bool_batch(
                self.ctx, n_inst, _ptr(nd, C.c_uint32), _ptr(eo, C.c_uint64), _ptr(s_, C.c_uint32),
                _ptr(d_, C.c_uint32), mode, _ptr(counts, C.c_uint64), _ptr(fps, C.c_uint64),
                _ptr(rounds, C.c_uint32), C.byref(st)))
        return BatchResult(counts, fps, rounds, st.as_dict())

    # -- Prov_k capture and provenance circuits -----------------------------
    def prov_capture(self, n_nodes: int, src, dst, prob, qs, qt, k: int = 8) -> "ProofSets":
        """Prov_k(k) proofs of path(s, t) for the query pairs (qs[q], qt[q]) of
        path(X,Y) :- edge(X,Y). path(X,Z) :- edge(X,Y), path(Y,Z). where edge
        i is the leaf with literal i+1 and probability prob[i] (FP64).
        src/dst/prob: device tensors or host arrays; qs/qt host arrays."""
        import torch
        if not hasattr(src, "data_ptr"):
            src = torch.from_numpy(_u32(src).view(np.int32)).cuda()
            dst = torch.from_numpy(_u32(dst).view(np.int32)).cuda()
        if not hasattr(prob, "data_ptr"):
            prob = torch.from_numpy(np.ascontiguousarray(prob, dtype=np.float64)).cuda()
        if prob.dtype != torch.float64:
            raise InvalidArgument("edge probabilities must be float64 (the FP64 of each input value)")
        qs_, qt_ = _u32(qs), _u32(qt)
        m = _len(src)
        if _len(dst) != m or _len(prob) != m:
            raise InvalidArgument("src, dst and prob must have one entry per edge")
        if len(qs_) != len(qt_):
            raise InvalidArgument("qs and qt must have the same length")
        out = C.c_void_p()
        st = L.ProvStats()
        rounds = np.zeros(max(1, len(np.unique(qt_))), np.uint32)
        self._check(self.lib.strata_prov_tc_capture(
            self.ctx, n_nodes, _dp(src), _dp(dst), m, _dp(prob), k, len(qs_), _ptr(qs_, C.c_uint32),
            _ptr(qt_, C.c_uint32), C.byref(out), _ptr(rounds, C.c_uint32), C.byref(st)))
        try:
            nq, np_, nl = C.c_uint32(), C.c_uint64(), C.c_uint64()
            self._check(self.lib.strata_proofs_shape(out, C.byref(nq), C.byref(np_), C.byref(nl)))
            po = np.zeros(nq.value + 1, np.uint64)
            lo = np.zeros(np_.value + 1, np.uint64)
            lits = np.zeros(max(1, nl.value), np.int64)
            self._check(self.lib.strata_proofs_export(out, _ptr(po, C.c_uint64), _ptr(lo, C.c_uint64),
                                                      _ptr(lits, C.c_int64)))
        finally:
            self.lib.strata_proofs_free(out)
        return ProofSets(po, lo, lits, st.as_dict(), rounds[:len(np.unique(qt_))])

    def compile_circuits(self, proofs, n_leaves: int, max_nodes: int = 0) -> "Circuits":
        """Exact circuits of each query's proof DNF (a ProofSets, or a list of
        lists of signed-literal lists)."""
        if not isinstance(proofs, ProofSets):
            proofs = ProofSets.from_lists(proofs)
        out = C.c_void_p()
        self._check(self.lib.strata_circuits_compile(
            self.ctx, len(proofs), _ptr(proofs.proof_off, C.c_uint64), _ptr(proofs.lit_off, C.c_uint64),
            _ptr(proofs.lits, C.c_int64), n_leaves, max_nodes, C.byref(out)))
        return Circuits(self, out, len(proofs), n_leaves)

    def compile_circuits_host(self, proofs, n_leaves: int, max_nodes: int = 0) -> "CircuitParts":
        """Host half of compile_circuits (no device work, usable from another
        thread while this engine runs a capture)."""
        if not isinstance(proofs, ProofSets):
            proofs = ProofSets.from_lists(proofs)
        out = C.c_void_p()
        rc = self.lib.strata_circuits_compile_host(
            len(proofs), _ptr(proofs.proof_off, C.c_uint64), _ptr(proofs.lit_off, C.c_uint64),
            _ptr(proofs.lits, C.c_int64), n_leaves, max_nodes, C.byref(out))
        if rc != L.OK:
            _raise(rc, self.lib.strata_circuit_parts_error().decode(errors="replace"))
        return CircuitParts(self.lib, out, len(proofs))

    def upload_circuits(self, parts, n_leaves: int) -> "Circuits":
        """Concatenate host-compiled parts (queries in part order) on the device."""
        arr = (C.c_void_p * max(1, len(parts)))(*[p.h for p in parts])
        out = C.c_void_p()
        self._check(self.lib.strata_circuits_upload(self.ctx, len(parts), arr, n_leaves, C.byref(out)))
        return Circuits(self, out, sum(p.n_queries for p in parts), n_leaves)

    def grad_queries(self, n_nodes: int, src, dst, prob64, prob32, qs, qt, k: int = 8, chunks: int = 4):
        """`?grad path(s, t)` for every query pair: Prov_k capture, exact
        compilation and the per-query gradient rows.  The queries are taken in
        `chunks` groups; while the device captures group i+1, a host thread
        compiles group i.  Returns (P [FP32, n_queries], G [FP64, n_queries x
        n_edges], Circuits, info)."""
        import queue
        import threading
        import time as _time
        qs_, qt_ = _u32(qs), _u32(qt)
        nq, m = len(qs_), _len(src)
        bounds = [nq * i // max(1, chunks) for i in range(max(1, chunks) + 1)]
        parts = [None] * max(1, chunks)
        todo: queue.Queue = queue.Queue()
        errors = []

        def compile_worker():
            while True:
                item = todo.get()
                if item is None:
                    return
                i, pr = item
                try:
                    parts[i] = self.compile_circuits_host(pr, m)
                except Exception as e:  # reported after the join
                    errors.append(e)

        worker = threading.Thread(target=compile_worker, daemon=True)
        worker.start()
        t0 = _time.perf_counter()
        stats = []
        try:
            for i in range(len(parts)):
                a, b = bounds[i], bounds[i + 1]
                pr = self.prov_capture(n_nodes, src, dst, prob64, qs_[a:b], qt_[a:b], k=k)
                stats.append(pr.stats)
                todo.put((i, pr))
        finally:
            todo.put(None)
            worker.join()
        if errors:
            raise errors[0]
        t1 = _time.perf_counter()
        circ = self.upload_circuits(parts, m)
        for part in parts:
            part.free()
        P = circ.forward(prob32)
        G = circ.grads(prob32)
        info = {"capture_and_compile_s": t1 - t0, "rounds_max": max((s_["rounds_max"] for s_ in stats), default=0),
                "max_proof_len": max((s_["max_proof_len"] for s_ in stats), default=0),
                "capture_device_ms": sum(s_["device_ms"] for s_ in stats), "chunks": len(parts)}
        return P, G, circ, info

    def asp_simplify_filter(self, head, body_start, body_lit, poss, cert):
        """``simplify_filter`` (strata-gpu/src/asp.rs:121) on the device:
        (head, body_start, body_lit) of the rules that survive, literals
        trimmed."""
        h = np.ascontiguousarray(head, np.int32)
        bs = np.ascontiguousarray(body_start, np.uint32)
        bl = np.ascontiguousarray(body_lit, np.int32)
        ps = np.ascontiguousarray(poss, np.uint8)
        ce = np.ascontiguousarray(cert, np.uint8)
        oh, ob, ol = C.POINTER(C.c_int32)(), C.POINTER(C.c_uint32)(), C.POINTER(C.c_int32)()
        n = C.c_uint64()
        self._check(self.lib.strata_asp_simplify_filter(
            self.ctx, len(h), _ptr(h, C.c_int32), _ptr(bs, C.c_uint32), _ptr(bl, C.c_int32), len(ps),
            _ptr(ps, C.c_uint8), _ptr(ce, C.c_uint8), C.byref(oh), C.byref(ob), C.byref(ol), C.byref(n)))
        m = n.value
        start = self._take(ob, m + 1, np.uint32)
        return self._take(oh, m, np.int32), start, self._take(ol, int(start[-1]), np.int32)

    def count_triangle_pattern_range_dev(self, x, y, x_lo: int, x_hi: int, n=None) -> int:
        """Bindings of the triangle pattern with X in [x_lo, x_hi)."""
        n = _len(x) if n is None else n
        out = C.c_uint64()
        self._check(self.lib.strata_count_triangle_pattern_range_dev(self.ctx, _dp(x), _dp(y), n, x_lo, x_hi,
                                                                     C.byref(out)))
        return int(out.value)

    def count_triangle_pattern_dev(self, x, y, n=None) -> int:
        n = _len(x) if n is None else n
        out = C.c_uint64()
        self._check(self.lib.strata_count_triangle_pattern_dev(self.ctx, _dp(x), _dp(y), n, C.byref(out)))
        return int(out.value)


def _dp(t) -> C.c_void_p | None:
    """Device pointer of a torch tensor (or an int), None for None."""
    if t is None:
        return None
    if isinstance(t, int):
        return C.c_void_p(t)
    return C.c_void_p(t.data_ptr())


def _len(t) -> int:
    return int(t.numel()) if hasattr(t, "numel") else len(t)


class ProofSets:
    """Flattened per-query proof sets: query q owns proofs
    [proof_off[q], proof_off[q+1]), proof p the literals [lit_off[p], lit_off[p+1])."""

    def __init__(self, proof_off, lit_off, lits, stats=None, target_rounds=None):
        self.proof_off = np.ascontiguousarray(proof_off, np.uint64)
        self.lit_off = np.ascontiguousarray(lit_off, np.uint64)
        self.lits = np.ascontiguousarray(lits, np.int64)
        if len(self.lits) == 0:
            self.lits = np.zeros(1, np.int64)
        self.stats = stats or {}
        self.target_rounds = target_rounds

    @staticmethod
    def from_lists(qs) -> "ProofSets":
        po, lo, lits = [0], [0], []
        for q in qs:
            for p in q:
                lits += [int(x) for x in p]
                lo.append(len(lits))
            po.append(len(lo) - 1)
        return ProofSets(po, lo, lits)

    def __len__(self) -> int:
        return len(self.proof_off) - 1

    def query(self, q: int) -> list:
        a, b = int(self.proof_off[q]), int(self.proof_off[q + 1])
        return [self.lits[int(self.lit_off[p]):int(self.lit_off[p + 1])].tolist() for p in range(a, b)]

    def as_lists(self) -> list:
        return [self.query(q) for q in range(len(self))]


class CircuitParts:
    """Host-compiled circuits of a group of queries (not yet on the device)."""

    def __init__(self, lib, handle, n_queries: int):
        self.lib, self.h, self.n_queries = lib, handle, n_queries

    def shape(self) -> tuple[int, int]:
        nq, nn, lv = C.c_uint32(), C.c_uint64(), C.c_uint32()
        rc = self.lib.strata_circuit_parts_shape(self.h, C.byref(nq), C.byref(nn), C.byref(lv))
        if rc != L.OK:
            _raise(rc, "invalid circuit parts")
        return int(nn.value), int(lv.value)

    def eval64(self, prob) -> np.ndarray:
        """FP64 P per query on the host (a check of the compiler)."""
        pr = np.ascontiguousarray(prob, np.float64)
        out = np.zeros(max(1, self.n_queries), np.float64)
        rc = self.lib.strata_circuit_parts_eval64(self.h, _ptr(pr, C.c_double), _ptr(out, C.c_double))
        if rc != L.OK:
            _raise(rc, "invalid circuit parts")
        return out[:self.n_queries]

    def free(self):
        if self.h:
            self.lib.strata_circuit_parts_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Circuits:
    """Compiled provenance circuits on the device (forward WMC, VJP, per-query grads)."""

    def __init__(self, eng: Engine, handle, n_queries: int, n_leaves: int):
        self.eng, self.h, self.n_queries, self.n_leaves = eng, handle, n_queries, n_leaves

    def shape(self) -> tuple[int, int]:
        n, lv = C.c_uint64(), C.c_uint32()
        self.eng._check(self.eng.lib.strata_circuits_shape(self.h, C.byref(n), C.byref(lv)))
        return int(n.value), int(lv.value)

    def forward(self, p, out64: bool = False):
        """P per query for FP32 leaf probabilities p (a CUDA tensor)."""
        import torch
        out = torch.empty(self.n_queries, dtype=torch.float64 if out64 else torch.float32, device=p.device)
        after = self.eng.on_torch_stream()
        self.eng._check(self.eng.lib.strata_circuits_forward(
            self.eng.ctx, self.h, _dp(p), None if out64 else _dp(out), _dp(out) if out64 else None))
        if after:
            self.eng.synchronize()
        return out

    def vjp(self, p, seed=None):
        """Σ_q seed[q] · dP_q/dp (FP32 tensor of n_leaves; FP64 accumulation)."""
        import torch
        g64 = torch.empty(max(1, self.n_leaves), dtype=torch.float64, device=p.device)
        g32 = torch.empty(max(1, self.n_leaves), dtype=torch.float32, device=p.device)
        after = self.eng.on_torch_stream()
        self.eng._check(self.eng.lib.strata_circuits_vjp(self.eng.ctx, self.h, _dp(p), _dp(seed), _dp(g64),
                                                         _dp(g32)))
        if after:
            self.eng.synchronize()
        return g32[:self.n_leaves], g64[:self.n_leaves]

    def grads(self, p):
        """[n_queries, n_leaves] FP64 per-query gradients (the ?grad rows)."""
        import torch
        g = torch.empty((max(1, self.n_queries), max(1, self.n_leaves)), dtype=torch.float64, device=p.device)
        after = self.eng.on_torch_stream()
        self.eng._check(self.eng.lib.strata_circuits_grads(self.eng.ctx, self.h, _dp(p), _dp(g)))
        if after:
            self.eng.synchronize()
        return g[:self.n_queries, :self.n_leaves]

    def free(self):
        if self.h:
            self.eng.lib.strata_circuits_free(self.eng.ctx, self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _torch_sync(*tensors):
    """Finish torch's queued work on the tensors' device before the engine's
    own stream reads them (the engine returns only after its stream is idle)."""
    import torch
    for t in tensors:
        if hasattr(t, "is_cuda") and t.is_cuda:
            torch.cuda.current_stream(t.device).synchronize()
            return


class TcShard:
    """One rank's share of a sharded Bool closure (``strata_tc_shard``):
    path rows [lo, hi) of n, ``per`` rows per rank, bit rows of
    ``row_bytes`` bytes.  Δ slices are int32 device tensors of
    per * row_bytes / 4 words, row flags uint8 tensors of ``per`` bytes."""

    def __init__(self, eng: Engine, handle, rank: int, world: int, keep=()):
        self.eng, self.h, self.rank, self.world = eng, handle, rank, world
        self._keep = keep  # the edge columns stay alive until the seed has read them
        per, lo, hi, rb = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64()
        eng._check(eng.lib.strata_tc_shard_shape(handle, C.byref(per), C.byref(lo), C.byref(hi), C.byref(rb)))
        self.per, self.lo, self.hi, self.row_bytes = int(per.value), int(lo.value), int(hi.value), int(rb.value)

    def shape(self) -> tuple[int, int, int, int]:
        return self.per, self.lo, self.hi, self.row_bytes

    def seed(self, mine, fmine) -> int:
        n = C.c_uint64()
        _torch_sync(mine)
        self.eng._check(self.eng.lib.strata_tc_shard_seed(self.eng.ctx, self.h, _dp(mine), _dp(fmine), C.byref(n)))
        self._keep = ()
        return int(n.value)

    def round(self, full, ffull, mine, fmine) -> int:
        n = C.c_uint64()
        _torch_sync(full)
        self.eng._check(self.eng.lib.strata_tc_shard_round(self.eng.ctx, self.h, _dp(full), _dp(ffull), _dp(mine),
                                                           _dp(fmine), C.byref(n)))
        return int(n.value)

    def summary(self) -> tuple[int, int]:
        c, f = C.c_uint64(), C.c_uint64()
        self.eng._check(self.eng.lib.strata_tc_shard_summary(self.eng.ctx, self.h, C.byref(c), C.byref(f)))
        return int(c.value), int(f.value)

    def pack_count(self, mine) -> int:
        """Nonzero 128-bit words of this rank's Δ' slice."""
        n = C.c_uint64()
        _torch_sync(mine)
        self.eng._check(self.eng.lib.strata_tc_shard_pack(self.eng.ctx, self.h, _dp(mine), None, 0, C.byref(n)))
        return int(n.value)

    def pack(self, mine, cap: int):
        """(cap, 3) int64 device tensor of (global word index, low, high)
        triples of the slice's nonzero words, padded with index -1."""
        import torch
        out = torch.empty((max(cap, 1), 3), dtype=torch.int64, device=mine.device)
        n = C.c_uint64()
        _torch_sync(mine)
        self.eng._check(self.eng.lib.strata_tc_shard_pack(self.eng.ctx, self.h, _dp(mine), _dp(out), cap,
                                                          C.byref(n)))
        if int(n.value) > cap:
            raise InvalidArgument(f"{int(n.value)} nonzero words exceed the capacity {cap}")
        return out[:cap]

    def unpack(self, triples, full, ffull):
        """Rebuild the gathered Δ and its row flags from all ranks' triples."""
        _torch_sync(triples)
        self.eng._check(self.eng.lib.strata_tc_shard_unpack(self.eng.ctx, self.h, _dp(triples), triples.shape[0],
                                                            _dp(full), _dp(ffull)))

    def free(self):
        if self.h:
            self.eng.lib.strata_tc_shard_free(self.h)
            self.h = None


class BatchResult:
    """Per-instance closure summaries of a batched call."""

    def __init__(self, counts, fps, rounds, stats):
        self.counts, self.fps, self.rounds, self.stats = counts, fps, rounds, stats

    def __len__(self) -> int:
        return len(self.counts)


class DeviceRelation:
    """A fixpoint result held on the device (``strata_rel``)."""

    def __init__(self, eng: Engine, rel, stats: dict):
        self.eng, self.rel, self.stats = eng, rel, stats

    def __len__(self) -> int:
        n = C.c_uint64()
        self.eng._check(self.eng.lib.strata_rel_size(self.rel, C.byref(n)))
        return int(n.value)

    @property
    def is_trop(self) -> bool:
        t = C.c_int()
        self.eng._check(self.eng.lib.strata_rel_is_trop(self.rel, C.byref(t)))
        return bool(t.value)

    def fingerprint(self) -> int:
        fp = C.c_uint64()
        self.eng._check(self.eng.lib.strata_rel_fingerprint(self.eng.ctx, self.rel, C.byref(fp)))
        return int(fp.value)

    def to_host(self, out=None):
        """Copy out; ``out`` may supply (pinned) numpy arrays to copy into."""
        n = len(self)
        trop = self.is_trop
        if out is None:
            s = np.zeros(n, np.uint32)
            d = np.zeros(n, np.uint32)
            w = np.zeros(n, np.int64) if trop else None
            i = np.zeros(n, np.uint8) if trop else None
        else:
            s, d, w, i = out
        self.eng._check(self.eng.lib.strata_rel_to_host(
            self.eng.ctx, self.rel, _ptr(s, C.c_uint32), _ptr(d, C.c_uint32),
            _ptr(w, C.c_int64) if w is not None else None, _ptr(i, C.c_uint8) if i is not None else None))
        if trop:
            return TropRelation(s[:n], d[:n], w[:n], i[:n], dict(self.stats))
        return BoolRelation(s[:n], d[:n], dict(self.stats))

    def free(self):
        if self.rel:
            self.eng.lib.strata_rel_free(self.eng.ctx, self.rel)
            self.rel = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---- module-level functions with the reference's names -----------------------
_default: dict[int, Engine] = {}
_dlock = threading.Lock()


def default_engine(device: int = 0) -> Engine:
    """A process-wide engine per device (the reference keeps one `CudaDevice`
    per module in a OnceLock, strata-gpu/src/sort.rs:221-254)."""
    with _dlock:
        if device not in _default:
            _default[device] = Engine(device)
        return _default[device]


def transitive_closure_bool(edges) -> BoolRelation:
    return default_engine().transitive_closure_bool(edges)


def shortest_paths_trop(edges) -> TropRelation:
    return default_engine().shortest_paths_trop(edges)


def mssp_trop(sources, edges, source_weights=None) -> TropRelation:
    return default_engine().mssp_trop(sources, edges, source_weights)


def count_triangles(edges) -> int:
    return default_engine().count_triangles(edges)


def count_4cliques(edges) -> int:
    return default_engine().count_4cliques(edges)


def count_triangle_pattern(edges) -> int:
    return default_engine().count_triangle_pattern(edges)


def intern_terms(keys) -> np.ndarray:
    return default_engine().intern_terms(keys)


def binary_plan_intermediate(edges) -> int:
    return default_engine().binary_plan_intermediate(edges)
