"""ctypes binding of ``libstrata_b200.so`` (the C ABI in include/strata_b200.h).

The shared library is built in-tree by ``strata-k_b200/build.py``.  Loading
fails loudly when it is missing: there is no CPU fallback anywhere in this
package.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libstrata_b200.so"

# strata_status codes (include/strata_b200.h)
OK = 0
E_INVALID = 1
E_OOM = 2
E_CUDA = 3
E_OVERFLOW = 4
E_NEG_CYCLE = 5
E_TIMEOUT = 6
E_UNSUPPORTED = 7
E_NOT_BUILT = 8
E_WEIGHT_RANGE = 9

PLAN_AUTO, PLAN_SORT_MERGE, PLAN_DENSE, PLAN_BITS = 0, 1, 2, 3
KNOB_SORT_ITEMS_U32, KNOB_SORT_ITEMS_U64, KNOB_TRI_PROBE = 1, 2, 3
KNOB_BATCH_GRAPH_ROUNDS, KNOB_BATCH_BLOCKS_PER_SM, KNOB_BATCH_BUDGET_MB = 4, 5, 6
KNOB_SORT_RANK = 7
KNOB_DENSE_WORD_MEMBERS = 8
KNOB_WEIGHT_LANES = 9

KERNELS = {0: "k_onesweep", 1: "k_expand_emit", 2: "k_expand_offsets", 3: "k_reduce_runs",
           4: "k_merge_diff", 5: "k_radix_hist", 6: "k_tri_count", 7: "k_expand_dense",
           8: "k_bs_round", 9: "k_prov_round", 10: "k_circuit", 11: "k_shard_round"}

STATUS_NAMES = {
    OK: "OK", E_INVALID: "INVALID", E_OOM: "OOM", E_CUDA: "CUDA", E_OVERFLOW: "OVERFLOW",
    E_NEG_CYCLE: "NEG_CYCLE", E_TIMEOUT: "TIMEOUT", E_UNSUPPORTED: "UNSUPPORTED",
    E_NOT_BUILT: "NOT_BUILT", E_WEIGHT_RANGE: "WEIGHT_RANGE",
}


class FixStats(C.Structure):
    """Mirror of ``strata_fix_stats``."""

    _fields_ = [
        ("rounds", C.c_uint64), ("candidates", C.c_uint64), ("result_tuples", C.c_uint64),
        ("universe", C.c_uint64), ("key_bits", C.c_uint32), ("weight_bytes", C.c_uint32),
        ("device_ms", C.c_double), ("sort_ms", C.c_double), ("join_ms", C.c_double),
        ("diff_ms", C.c_double), ("merge_ms", C.c_double),
        ("sort_bytes", C.c_uint64), ("join_bytes", C.c_uint64), ("diff_bytes", C.c_uint64),
        ("merge_bytes", C.c_uint64),
        ("sort_launches", C.c_uint32), ("join_launches", C.c_uint32),
        ("diff_launches", C.c_uint32), ("merge_launches", C.c_uint32),
        ("other_launches", C.c_uint32), ("plan", C.c_uint32),
        ("setup_ms", C.c_double), ("finish_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchStats(C.Structure):
    """Mirror of ``strata_batch_stats``."""

    _fields_ = [
        ("instances", C.c_uint64), ("waves", C.c_uint64), ("graph_launches", C.c_uint64),
        ("round_launches", C.c_uint64), ("rounds_max", C.c_uint64), ("result_tuples", C.c_uint64),
        ("round_bytes", C.c_uint64), ("launches", C.c_uint64), ("device_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class ProvStats(C.Structure):
    """Mirror of ``strata_prov_stats``."""

    _fields_ = [
        ("queries", C.c_uint64), ("targets", C.c_uint64), ("waves", C.c_uint64), ("rounds_max", C.c_uint64),
        ("max_proof_len", C.c_uint64), ("launches", C.c_uint64), ("device_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
i64p = C.POINTER(C.c_int64)
vp = C.c_void_p
ctxp = C.c_void_p
relp = C.c_void_p

# Every exported symbol with (restype, argtypes); the CPU tests check that the
# library exports exactly these names.
SIGNATURES = {
    "strata_version": (C.c_char_p, []),
    "strata_ctx_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(ctxp)]),
    "strata_ctx_destroy": (None, [ctxp]),
    "strata_ctx_set_stream": (C.c_int, [ctxp, vp]),
    "strata_ctx_synchronize": (C.c_int, [ctxp]),
    "strata_last_error": (C.c_char_p, [ctxp]),
    "strata_ctx_mem": (C.c_int, [ctxp, u64p, u64p]),
    "strata_ctx_set_profiling": (C.c_int, [ctxp, C.c_int]),
    "strata_ctx_set_plan": (C.c_int, [ctxp, C.c_int]),
    "strata_ctx_set_knob": (C.c_int, [ctxp, C.c_int, C.c_int]),
    "strata_tc_bool_batch_dev": (C.c_int, [ctxp, C.c_uint32, u32p, u64p, vp, vp, C.c_int, u64p, u64p, u32p,
                                           C.POINTER(BatchStats)]),
    "strata_tc_bool_batch": (C.c_int, [ctxp, C.c_uint32, u32p, u64p, u32p, u32p, C.c_int, u64p, u64p, u32p,
                                       C.POINTER(BatchStats)]),
    "strata_tc_shard_create": (C.c_int, [ctxp, C.c_uint32, vp, vp, C.c_uint64, C.c_uint32, C.c_uint32,
                                         C.POINTER(vp)]),
    "strata_tc_shard_shape": (C.c_int, [vp, u32p, u32p, u32p, u64p]),
    "strata_tc_shard_seed": (C.c_int, [ctxp, vp, vp, vp, u64p]),
    "strata_tc_shard_round": (C.c_int, [ctxp, vp, vp, vp, vp, vp, u64p]),
    "strata_tc_shard_summary": (C.c_int, [ctxp, vp, u64p, u64p]),
    "strata_tc_shard_pack": (C.c_int, [ctxp, vp, vp, vp, C.c_uint64, u64p]),
    "strata_tc_shard_unpack": (C.c_int, [ctxp, vp, vp, C.c_uint64, vp, vp]),
    "strata_tc_shard_free": (None, [vp]),
    "strata_prov_tc_capture": (C.c_int, [ctxp, C.c_uint32, vp, vp, C.c_uint64, vp, C.c_uint32, C.c_uint32, u32p,
                                         u32p, C.POINTER(vp), u32p, C.POINTER(ProvStats)]),
    "strata_proofs_shape": (C.c_int, [vp, u32p, u64p, u64p]),
    "strata_proofs_export": (C.c_int, [vp, u64p, u64p, i64p]),
    "strata_proofs_free": (None, [vp]),
    "strata_circuits_compile": (C.c_int, [ctxp, C.c_uint32, u64p, u64p, i64p, C.c_uint32, C.c_uint64,
                                          C.POINTER(vp)]),
    "strata_circuits_shape": (C.c_int, [vp, u64p, u32p]),
    "strata_count_triangle_pattern_range_dev": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.c_uint64, C.c_uint64, u64p]),
    "strata_circuits_compile_host": (C.c_int, [C.c_uint32, u64p, u64p, i64p, C.c_uint32, C.c_uint64,
                                               C.POINTER(vp)]),
    "strata_circuit_parts_error": (C.c_char_p, []),
    "strata_circuits_upload": (C.c_int, [ctxp, C.c_uint32, C.POINTER(vp), C.c_uint32, C.POINTER(vp)]),
    "strata_circuit_parts_free": (None, [vp]),
    "strata_circuit_parts_shape": (C.c_int, [vp, u32p, u64p, u32p]),
    "strata_circuit_parts_eval64": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "strata_circuits_forward": (C.c_int, [ctxp, vp, vp, vp, vp]),
    "strata_circuits_vjp": (C.c_int, [ctxp, vp, vp, vp, vp, vp]),
    "strata_circuits_grads": (C.c_int, [ctxp, vp, vp, vp]),
    "strata_circuits_free": (None, [ctxp, vp]),
    "strata_ctx_launches": (C.c_uint64, [ctxp]),
    "strata_ctx_kernel_stats": (C.c_int, [ctxp, C.c_int, u64p, C.POINTER(C.c_double), u64p]),
    "strata_ctx_reset_kernel_stats": (C.c_int, [ctxp]),
    "strata_free": (None, [vp]),
    "strata_transitive_closure_bool": (
        C.c_int, [ctxp, u32p, u32p, C.c_uint64, C.POINTER(u32p), C.POINTER(u32p), u64p,
                  C.POINTER(FixStats)]),
    "strata_shortest_paths_trop": (
        C.c_int, [ctxp, u32p, u32p, i64p, u8p, C.c_uint64, C.POINTER(u32p), C.POINTER(u32p),
                  C.POINTER(i64p), C.POINTER(u8p), u64p, C.POINTER(FixStats)]),
    "strata_mssp_trop": (
        C.c_int, [ctxp, u32p, i64p, u8p, C.c_uint64, u32p, u32p, i64p, u8p, C.c_uint64,
                  C.POINTER(u32p), C.POINTER(u32p), C.POINTER(i64p), C.POINTER(u8p), u64p,
                  C.POINTER(FixStats)]),
    "strata_count_triangles": (C.c_int, [ctxp, u32p, u32p, C.c_uint64, u64p]),
    "strata_count_4cliques": (C.c_int, [ctxp, u32p, u32p, C.c_uint64, u64p]),
    "strata_count_triangle_pattern": (C.c_int, [ctxp, u32p, u32p, C.c_uint64, u64p]),
    "strata_intern_terms": (C.c_int, [ctxp, u64p, C.c_uint64, u32p, u64p]),
    "strata_binary_plan_intermediate": (C.c_int, [ctxp, u32p, u32p, C.c_uint64, u64p]),
    "strata_tc_bool_dev": (C.c_int, [ctxp, vp, vp, C.c_uint64, C.POINTER(relp), C.POINTER(FixStats)]),
    "strata_trop_paths_dev": (
        C.c_int, [ctxp, vp, vp, vp, vp, C.c_uint64, C.POINTER(relp), C.POINTER(FixStats)]),
    "strata_mssp_trop_dev": (
        C.c_int, [ctxp, vp, vp, vp, C.c_uint64, vp, vp, vp, vp, C.c_uint64, C.POINTER(relp),
                  C.POINTER(FixStats)]),
    "strata_count_triangle_pattern_dev": (C.c_int, [ctxp, vp, vp, C.c_uint64, u64p]),
    "strata_rel_size": (C.c_int, [relp, u64p]),
    "strata_rel_is_trop": (C.c_int, [relp, C.POINTER(C.c_int)]),
    "strata_rel_to_host": (C.c_int, [ctxp, relp, u32p, u32p, i64p, u8p]),
    "strata_rel_fingerprint": (C.c_int, [ctxp, relp, u64p]),
    "strata_rel_free": (None, [ctxp, relp]),
    "strata_op_sort": (C.c_int, [ctxp, C.c_int, C.c_int, vp, vp, vp, vp, C.c_uint64, C.c_int]),
    "strata_op_dedup_diff": (C.c_int, [ctxp, C.c_int, vp, C.c_uint64, vp, C.c_uint64, vp, u64p]),
    "strata_op_min_improve": (
        C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, vp, vp, C.c_uint64, vp, vp, u64p]),
    "strata_op_merge": (C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, vp, vp, C.c_uint64, vp, vp]),
    "strata_op_reduce": (C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, vp, vp, C.POINTER(C.c_uint64)]),
    "strata_op_merge_diff": (C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, vp, vp, C.c_uint64, vp, vp, vp, vp,
                                       C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "strata_op_select": (C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, C.c_int, C.c_int, C.c_uint64, vp, vp,
                                   C.POINTER(C.c_uint64)]),
    "strata_op_intersect": (C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, vp, vp, C.c_uint64, vp, vp,
                                      C.POINTER(C.c_uint64)]),
    "strata_op_semijoin": (C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, vp, vp, C.c_uint64, C.c_int, vp, vp,
                                     C.POINTER(C.c_uint64)]),
    "strata_asp_simplify_filter": (C.c_int, [ctxp, C.c_uint64, vp, vp, vp, C.c_uint64, vp, vp,
                                             C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_uint32)),
                                             C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.c_uint64)]),
    "strata_tsv_load": (C.c_int, [ctxp, C.c_char_p, C.c_uint64, C.c_uint32, C.c_int, C.c_char_p, vp, C.c_uint64,
                                  C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.POINTER(C.c_int64)),
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_void_p), C.POINTER(C.POINTER(C.c_uint64)),
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "strata_rel_render": (C.c_int, [ctxp, vp, C.c_char_p, C.c_char_p, vp, C.c_uint64, C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_uint64)]),
    "strata_op_join": (C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, C.c_int, vp, vp, C.c_uint64, C.c_int, C.c_int,
                                 vp, vp, C.c_uint64, C.POINTER(C.c_uint64)]),
    "strata_op_project": (C.c_int, [ctxp, C.c_int, vp, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                    C.c_uint64, C.c_int, C.c_int, vp]),
    "strata_op_aggregate": (C.c_int, [ctxp, C.c_int, vp, vp, C.c_uint64, C.c_int, C.c_int, vp, vp,
                                      C.POINTER(C.c_uint64)]),
    "strata_sort_u32_noalloc": (C.c_int, [vp, vp, C.c_uint64, C.c_int, vp]),
}

_lib = None
_lock = threading.Lock()


class LibraryMissing(RuntimeError):
    """The CUDA library was not built; the engine has no CPU path to fall back to."""


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the engine library once (fails loudly if it is missing)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            raise LibraryMissing(
                f"{p} not found: build it with `python strata-k_b200/build.py` "
                "(there is no CPU fallback)")
        lib = C.CDLL(str(p))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib
