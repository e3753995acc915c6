"""Parity at the full sizes of the benchmark configurations.

Each test runs the CUDA path (through the C ABI) on the same seeded workload
the benchmark times and compares it with the CPU oracle at that size:

  * Trop MSSP, R-MAT scale 20 (8,388,608 edges, i64 weights U[1,100],
    64 sources): every (S, Z, dist) row, bit-exact, against Dijkstra per
    source (both plans; with non-negative weights the fixpoint's minima are
    the shortest distances);
  * the triangle count on undirected R-MAT scale 22 (67,108,864 edges,
    oriented by degree): the exact count against a sorted-list intersection
    per edge;
  * 4,096 batched Bool closures: every instance's |path| and fingerprint
    against the SCC-condensation closure count;
  * Prov_k(8) reachability on ER(20,000, 80,000) with 1,024 (s, t) queries:
    proof sets of a spread sample of queries against the restated capture;
    P and every gradient entry of all 1,024 queries against the FP64 circuit
    oracle; the GPU gradient against central finite differences (h = 1e-3) of
    the FP64 evaluation of the same compiled circuit.

Integer results are exact.  The FP32 circuits are held to REL_TOL relative
error against FP64 (the reference evaluates in FP64, strata-prob/src/circuit.rs).
"""
import os

import numpy as np
import pytest

import oracle as O
from strata_b200 import gen

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)
REL_TOL = 1e-5


def _dev(a, dt):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).astype(dt)).cuda()


# ------------------------------------------------------------ C2: MSSP R-MAT-20
@pytest.fixture(scope="module")
def mssp20():
    wl = gen.mssp_workload(scale=20, n_sources=64, seed=2)
    want = O.dijkstra_mssp_rows(wl.sources, wl.src, wl.dst, wl.w, wl.source_w, threads=THREADS)
    return wl, want


@pytest.mark.parametrize("plan", [0, 1], ids=["auto", "sortmerge"])
def test_mssp_rmat20_64src_rows_equal_dijkstra(engine, mssp20, plan):
    wl, (ws, wd, ww) = mssp20
    engine.set_plan(plan)
    try:
        rel = engine.mssp_dev(_dev(wl.sources, np.int32), _dev(wl.src, np.int32), _dev(wl.dst, np.int32),
                              _dev(wl.w, np.int64), source_weights=_dev(wl.source_w, np.int64))
        try:
            assert len(rel) == len(ws)
            got = rel.to_host()
            assert np.array_equal(got.src, ws)
            assert np.array_equal(got.dst, wd)
            assert not got.inf.any()
            assert np.array_equal(got.w, ww)
            assert rel.stats["plan"] == (2 if plan == 0 else 1)
        finally:
            rel.free()
    finally:
        engine.set_plan(0)


# ------------------------------------------------------------ C3: triangles R-MAT-22
def test_triangle_pattern_rmat22_exact(engine):
    wl = gen.triangle_workload(scale=22, edge_factor=16, seed=3)
    assert len(wl.src) == 16 << 22
    want = O.count_pattern(wl.src, wl.dst, threads=THREADS)
    got = engine.count_triangle_pattern_dev(_dev(wl.src, np.int32), _dev(wl.dst, np.int32))
    assert got == want
    assert want > 0


# ------------------------------------------------------------ C4: 4,096 batched closures
def test_batch_4096_instances_every_instance_exact(engine):
    wl = gen.batch_tc_workload(n_inst=4096, seed=4, workers=min(16, THREADS))
    assert len(wl) == 4096
    counts, fps = O.closure_batch(wl.nodes, wl.edge_off, wl.src, wl.dst, threads=THREADS)
    res = engine.tc_bool_batch(wl.nodes, wl.edge_off, _dev(wl.src, np.int32), _dev(wl.dst, np.int32), mode=0)
    bad = np.flatnonzero((res.counts != counts) | (res.fps != fps))
    assert len(bad) == 0, f"{len(bad)} instances differ, first {bad[:8].tolist()}"
    assert res.stats["instances"] == 4096


# ------------------------------------------------------------ C5: Prov_k(8) ?grad, 1,024 queries
@pytest.fixture(scope="module")
def prov_full(engine):
    import torch
    wl = gen.prov_workload(n=20_000, m=80_000, n_queries=1024, seed=5)
    proofs = engine.prov_capture(wl.n, wl.src, wl.dst, wl.p64, wl.qs, wl.qt, k=8)
    circ = engine.compile_circuits(proofs, len(wl.src))
    pt = torch.from_numpy(wl.p32).cuda()
    P32 = circ.forward(pt).cpu().numpy().astype(np.float64)
    P64 = circ.forward(pt, out64=True).cpu().numpy()
    G = circ.grads(pt).cpu().numpy()  # [1024, 80000] FP64 rows of the FP32 adjoints
    circ.free()
    return wl, proofs, P32, P64, G


def test_prov_config_proof_sets_sample_equal_oracle(prov_full):
    """Exact top-8 proof sets for a spread sample of the 1,024 queries (the
    restated naive-round capture costs seconds per query on the host)."""
    wl, proofs, *_ = prov_full
    sample = np.arange(0, 1024, 16)  # 64 queries
    want, _ = O.prov_tc(wl.n, wl.src, wl.dst, wl.p64, 8, wl.qs[sample], wl.qt[sample], threads=THREADS)
    got = [proofs.query(int(q)) for q in sample]
    assert got == want


def test_prov_config_all_queries_p_and_every_gradient_entry_vs_fp64(prov_full):
    wl, proofs, P32, P64, G = prov_full
    worst_p, worst_leaf, n_leaf, nonzero = 0.0, 0.0, 0, 0
    for q in range(1024):
        want_p, want_g, _ = O.compile_grad(proofs.query(q), wl.p64)
        if want_p == 0.0:
            assert P32[q] == 0.0 and P64[q] == 0.0 and not G[q].any()
            continue
        nonzero += 1
        worst_p = max(worst_p, abs(P32[q] - want_p) / want_p, abs(P64[q] - want_p) / want_p)
        nz = want_g != 0.0
        assert not G[q][~nz].any(), q  # leaves outside the query's circuit get exactly 0
        rel = np.abs(G[q][nz] - want_g[nz]) / np.abs(want_g[nz])
        n_leaf += int(nz.sum())
        if len(rel):
            worst_leaf = max(worst_leaf, float(rel.max()))
    assert nonzero > 0
    print(f"queries with P > 0: {nonzero}; gradient entries checked: {n_leaf}; "
          f"max rel err P {worst_p:.3e}, per entry {worst_leaf:.3e}")
    assert worst_p <= REL_TOL
    assert worst_leaf <= REL_TOL


def test_prov_config_gpu_gradient_vs_central_differences(engine, prov_full):
    """dP/dp_i of the GPU adjoint against (P(p_i + h) - P(p_i - h)) / 2h of the
    FP64 evaluation of the same compiled circuit, h = 1e-3, on 32 leaves of
    every query (P is multilinear in each leaf, so the central difference is
    exact up to FP64 rounding)."""
    from strata_b200.gpu import ProofSets
    wl, proofs, P32, P64, G = prov_full
    h = 1e-3
    worst, checked = 0.0, 0
    for q in range(1024):
        pr = proofs.query(q)
        if not pr:
            continue
        leaves = sorted({abs(x) - 1 for p in pr for x in p})[:32]
        parts = engine.compile_circuits_host(ProofSets.from_lists([pr]), len(wl.src))
        try:
            for i in leaves:
                pp, pm = wl.p64.copy(), wl.p64.copy()
                pp[i] += h
                pm[i] -= h
                fd = (parts.eval64(pp)[0] - parts.eval64(pm)[0]) / (2 * h)
                err = abs(G[q, i] - fd) / max(abs(fd), 1e-300)
                worst = max(worst, err)
                checked += 1
        finally:
            parts.free()
    print(f"central differences: {checked} leaves, max rel err of the GPU gradient {worst:.3e}")
    assert checked >= 32
    assert worst <= REL_TOL
