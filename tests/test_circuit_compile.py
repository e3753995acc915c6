"""CPU checks of the engine's circuit compiler (host half of
strata_circuits_compile, no device needed) against the FP64 oracle's
restatement of compile_exact + Circuit::wmc (strata-prob/src/compile.rs,
circuit.rs): same node count per query and bit-identical FP64 values."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from strata_b200 import _lib as L
from strata_b200.gpu import CircuitParts, ProofSets


def _compile(lib, proofs, n_leaves):
    ps = ProofSets.from_lists(proofs)
    out = C.c_void_p()
    rc = lib.strata_circuits_compile_host(len(ps), ps.proof_off.ctypes.data_as(C.POINTER(C.c_uint64)),
                                          ps.lit_off.ctypes.data_as(C.POINTER(C.c_uint64)),
                                          ps.lits.ctypes.data_as(C.POINTER(C.c_int64)), n_leaves, 0, C.byref(out))
    return rc, CircuitParts(lib, out, len(ps)) if rc == 0 else None


@pytest.fixture(scope="module")
def lib():
    return L.load()


def test_compile_matches_oracle_random_dnfs(lib):
    rng = np.random.default_rng(11)
    queries, probs = [], rng.uniform(0.05, 0.95, 24)
    for _ in range(200):
        nproofs = int(rng.integers(0, 9))
        q = []
        for _ in range(nproofs):
            ln = int(rng.integers(0, 7))
            lits = rng.choice(np.arange(1, 25), ln, replace=False)
            sign = np.where(rng.random(ln) < 0.25, -1, 1)
            q.append(sorted(int(x) for x in lits * sign))
        queries.append(q)
    rc, parts = _compile(lib, queries, 24)
    assert rc == 0
    got = parts.eval64(probs)
    nodes = 0
    for i, q in enumerate(queries):
        want, _, nn = O.compile_grad(q, probs)
        assert got[i] == want, i  # same DAG, same fold order: bit-identical
        nodes += nn
    assert parts.shape()[0] == nodes
    parts.free()


def test_compile_rejects_bad_literal(lib):
    rc, _ = _compile(lib, [[[1, 30]]], 24)
    assert rc == L.E_INVALID
    assert b"leaf" in lib.strata_circuit_parts_error()
