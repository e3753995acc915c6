"""Prov_k capture, exact compilation and the FP32 circuit kernels against the
FP64 oracle (the restatement of strata-eval/src/provenance.rs and
strata-prob/src/{compile,circuit}.rs, pinned to the reference's AML lines)."""
import numpy as np
import pytest

import oracle as O
import strata_b200 as S
from strata_b200 import gen

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5  # FP32 circuits vs the FP64 oracle (relative)


def _probs(m, seed):
    """Beta(2,5) edge probabilities as fp32; the FP64 view is the same values."""
    p32 = np.random.default_rng(seed).beta(2.0, 5.0, m).astype(np.float32)
    return p32, p32.astype(np.float64)


def test_capture_matches_oracle_small_all_pairs(engine):
    rng = np.random.default_rng(3)
    for trial in range(25):
        n = int(rng.integers(3, 14))
        pairs = {(int(a), int(b)) for a, b in zip(rng.integers(0, n, 3 * n), rng.integers(0, n, 3 * n))}
        src = np.array([a for a, _ in sorted(pairs)], np.uint32)
        dst = np.array([b for _, b in sorted(pairs)], np.uint32)
        perm = rng.permutation(len(src))  # edge fact order = literal order
        src, dst = src[perm], dst[perm]
        _, p64 = _probs(len(src), trial)
        k = int(rng.integers(1, 9))
        qs = np.repeat(np.arange(n), n).astype(np.uint32)
        qt = np.tile(np.arange(n), n).astype(np.uint32)
        want, want_rounds = O.prov_tc(n, src, dst, p64, k, qs, qt, threads=4)
        got = engine.prov_capture(n, src, dst, p64, qs, qt, k=k)
        assert got.as_lists() == want, trial
        assert got.target_rounds.tolist() == [want_rounds[t] for t in sorted(want_rounds)]


def test_capture_matches_oracle_er_medium(engine):
    n, m = 3000, 12000
    s, d = gen.er_directed(n, m, 17)
    _, p64 = _probs(m, 18)
    rng = np.random.default_rng(19)
    qs = rng.integers(0, n, 48).astype(np.uint32)
    qt = rng.integers(0, n, 48).astype(np.uint32)
    want, _ = O.prov_tc(n, s, d, p64, 8, qs, qt, threads=8)
    got = engine.prov_capture(n, s, d, p64, qs, qt, k=8)
    assert got.as_lists() == want
    assert got.stats["max_proof_len"] <= 32


def test_capture_config_graph_sample(engine):
    """The differentiable-reachability graph itself (ER 20,000 / 80,000,
    Beta(2,5) fp32 probabilities), a sample of query pairs."""
    n, m = 20_000, 80_000
    s, d = gen.er_directed(n, m, 5)
    _, p64 = _probs(m, 6)
    rng = np.random.default_rng(7)
    qs = rng.integers(0, n, 6).astype(np.uint32)
    qt = rng.integers(0, n, 6).astype(np.uint32)
    want, _ = O.prov_tc(n, s, d, p64, 8, qs, qt, threads=8)
    got = engine.prov_capture(n, s, d, p64, qs, qt, k=8)
    assert got.as_lists() == want


def test_circuits_forward_and_grads_vs_fp64(engine):
    import torch
    n, m = 3000, 12000
    s, d = gen.er_directed(n, m, 21)
    p32, p64 = _probs(m, 22)
    rng = np.random.default_rng(23)
    qs = rng.integers(0, n, 64).astype(np.uint32)
    qt = rng.integers(0, n, 64).astype(np.uint32)
    proofs = engine.prov_capture(n, s, d, p64, qs, qt, k=8)
    circ = engine.compile_circuits(proofs, m)
    pt = torch.from_numpy(p32).cuda()
    P = circ.forward(pt).cpu().numpy().astype(np.float64)
    P64 = circ.forward(pt, out64=True).cpu().numpy()
    G = circ.grads(pt).cpu().numpy()
    worst_p, worst_g = 0.0, 0.0
    for q in range(len(qs)):
        want_p, want_g, _ = O.compile_grad(proofs.query(q), p64)
        if want_p == 0.0:
            assert P[q] == 0.0 and not G[q].any()
            continue
        worst_p = max(worst_p, abs(P64[q] - want_p) / want_p)
        assert abs(P[q] - want_p) <= REL_TOL * want_p
        nrm = np.linalg.norm(want_g)
        worst_g = max(worst_g, np.linalg.norm(G[q] - want_g) / nrm)
    assert worst_p <= REL_TOL and worst_g <= REL_TOL, (worst_p, worst_g)
    circ.free()


def test_autograd_function_matches_fd_and_vjp(engine):
    """torch.autograd backward = Σ_q seed_q ∂P_q/∂p; central differences
    (h = 1e-3) of the FP64 oracle agree (P is multilinear in each leaf)."""
    import torch

    from strata_b200.torch_bridge import prov_probability
    n, m = 1500, 6000
    s, d = gen.er_directed(n, m, 31)
    p32, p64 = _probs(m, 32)
    rng = np.random.default_rng(33)
    qs = rng.integers(0, n, 16).astype(np.uint32)
    qt = rng.integers(0, n, 16).astype(np.uint32)
    proofs = engine.prov_capture(n, s, d, p64, qs, qt, k=8)
    circ = engine.compile_circuits(proofs, m)
    pt = torch.from_numpy(p32).cuda().requires_grad_(True)
    w = torch.from_numpy(rng.uniform(0.5, 2.0, len(qs)).astype(np.float32)).cuda()
    P = prov_probability(pt, circ)
    (P * w).sum().backward()
    g = pt.grad.detach().cpu().numpy().astype(np.float64)
    want = np.zeros(m)
    wv = w.cpu().numpy().astype(np.float64)
    for q in range(len(qs)):
        want += wv[q] * O.compile_grad(proofs.query(q), p64)[1]
    nz = np.flatnonzero(want)
    if len(nz):
        assert np.linalg.norm(g - want) <= REL_TOL * np.linalg.norm(want)
    # finite differences on sampled leaves of each query (oracle FP64)
    h = 1e-3
    for q in range(len(qs)):
        pr = proofs.query(q)
        leaves = sorted({abs(x) - 1 for p in pr for x in p})[:32]
        _, gq, _ = O.compile_grad(pr, p64)
        for i in leaves:
            pp, pm = p64.copy(), p64.copy()
            pp[i] += h
            pm[i] -= h
            fd = (O.compile_grad(pr, pp)[0] - O.compile_grad(pr, pm)[0]) / (2 * h)
            assert abs(fd - gq[i]) <= 1e-9 + 1e-7 * abs(gq[i])
    circ.free()


def test_circuit_known_values(engine):
    """0.625 / d = 0.75 (strata-k/tests/facade.rs:38-52), DIAMOND 0.86 and
    dP/dp(ac) = 0.28 (strata-py/tests/test_bridge.py:42-54), 0.804
    (facade.rs:56-76): capture on the GPU, circuits on the GPU."""
    import torch
    cases = [
        ([(0, 2), (0, 1), (1, 2)], [0.5, 0.5, 0.5], 0.625, (0, 0.75)),
        ([(0, 1), (1, 2), (0, 2)], [0.9, 0.8, 0.5], 0.86, (2, 0.28)),
        ([(0, 1), (1, 2), (0, 2)], [0.9, 0.8, 0.3], 0.804, None),
    ]
    for edges, probs, want, gw in cases:
        src = np.array([a for a, _ in edges], np.uint32)
        dst = np.array([b for _, b in edges], np.uint32)
        p64 = np.array(probs, np.float64)
        pr = engine.prov_capture(3, src, dst, p64, [0], [2], k=8)
        circ = engine.compile_circuits(pr, 3)
        pt = torch.tensor(probs, dtype=torch.float32, device="cuda")
        assert abs(float(circ.forward(pt, out64=True)[0]) - want) < 1e-6
        if gw:
            assert abs(float(circ.grads(pt)[0, gw[0]]) - gw[1]) < 1e-6
        circ.free()


def test_capture_rejects_bad_input(engine):
    with pytest.raises(S.Unsupported):  # duplicate edge tuple
        engine.prov_capture(3, [0, 0], [1, 1], [0.5, 0.5], [0], [1])
    with pytest.raises(S.InvalidArgument):  # k out of range
        engine.prov_capture(3, [0], [1], [0.5], [0], [1], k=9)
    with pytest.raises(S.InvalidArgument):  # endpoint outside [0, n)
        engine.prov_capture(3, [0], [5], [0.5], [0], [1])
    with pytest.raises(S.InvalidArgument):  # query outside [0, n)
        engine.prov_capture(3, [0], [1], [0.5], [4], [1])


def test_grad_queries_pipeline_equals_direct(engine):
    """The chunked capture + host-compile pipeline gives the same P and
    gradient rows as one capture and one compilation."""
    import torch
    n, m = 1200, 4800
    s, d = gen.er_directed(n, m, 41)
    p32, p64 = _probs(m, 42)
    rng = np.random.default_rng(43)
    qs = rng.integers(0, n, 37).astype(np.uint32)
    qt = rng.integers(0, n, 37).astype(np.uint32)
    pt = torch.from_numpy(p32).cuda()
    P, G, circ, info = engine.grad_queries(n, s, d, p64, pt, qs, qt, k=8, chunks=5)
    pr = engine.prov_capture(n, s, d, p64, qs, qt, k=8)
    c2 = engine.compile_circuits(pr, m)
    assert torch.equal(P, c2.forward(pt))
    # node adjoints accumulate through FP32 atomics (and leaves through FP64
    # ones) whose order changes from launch to launch: equal up to FP32
    # rounding of the adjoints
    G2 = c2.grads(pt)
    assert torch.allclose(G, G2, rtol=1e-6, atol=1e-8), float((G - G2).abs().max())
    assert info["chunks"] == 5
    circ.free()
    c2.free()
