"""Pins the CPU oracle against the reference's own routines.

oracle/_ref/libkahip_ref.so is the reference KaHIP library compiled from its
sources (oracle/Makefile `ref`), with oracle/ref_harness.cpp exposing single
routines.  Where the deterministic schedule coincides with the reference's
(sequential node order, no ties), the oracle must reproduce the reference
bit for bit; everywhere else the oracle's building blocks (bounds, stop rule,
rating, contraction, metrics) must equal the reference's.

Skipped where the reference library was not built (no sources present);
tests/test_golden.py then checks the oracle against committed reference
outputs instead.
"""
import numpy as np
import pytest

from conftest import csr_from_edges, tie_free

from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference library (oracle/_ref) not built")


def _graph_set(graphs):
    rng = np.random.default_rng(0)
    g1 = graphs.rgg2d(3000, seed=1)
    g2 = graphs.rgg3d(2000, seed=2)
    g3 = graphs.rmat(11, seed=3)
    g4 = graphs.grid2d(40, 30)
    g5 = tie_free(graphs.rgg2d(2500, seed=4))
    g5["vwgt"] = rng.integers(1, 9, g5["n"]).astype(np.int32)
    return [g1, g2, g3, g4, g5]


@pytest.mark.parametrize("n,k,imb,mode", [(1 << 24, 64, 0.03, 0), (1 << 15, 8, 0.03, 1), (5000, 3, 0.0, 0),
                                          (777, 256, 0.05, 2), (100, 7, 0.1, 3), (1 << 20, 2, 0.001, 4)])
def test_balance_configuration_and_stop_rule(n, k, imb, mode):
    vw = None
    if n < 10000:
        vw = np.random.default_rng(n).integers(1, 5, n).astype(np.int32)
    U, ns, mv = O.ref_balance_config(n, vw, k, imb, mode)
    g = dict(n=n, vwgt=vw if vw is not None else np.ones(n, np.int32))
    kn = O.knobs(g, k, imb, 0, mode)
    assert (kn.upper_bound, kn.num_stop, kn.max_vertex_weight) == (U, ns, mv)
    W = int(g["vwgt"].sum())
    for nf, nc in [(n, n), (n, int(n / 1.1) + 1), (n, int(n / 1.1)), (10 * ns, ns), (10 * ns, ns - 1), (5, 1)]:
        if nc <= 0:
            continue
        assert O.stop_continue(kn, nf, nc) == O.ref_stop_continue(nf, nc, n, k, W)


def test_expansion_star_2_rating(graphs):
    for g in _graph_set(graphs):
        a = O.rating(g)
        b = O.ref_rating(g)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def _as_reference_int(cut2):
    """quality_metrics.cpp:23-37 sums directed entries in a 32-bit int and
    halves it; the oracle sums in 64 bits.  Reproduce the int arithmetic."""
    s = ((cut2 + (1 << 31)) % (1 << 32)) - (1 << 31)
    return int(s / 2)


def test_edge_cut_and_balance(graphs):
    rng = np.random.default_rng(1)
    for g in _graph_set(graphs):
        for k in (2, 5, 64):
            part = rng.integers(0, k, g["n"]).astype(np.int32)
            cut = O.edge_cut(g, part)
            assert _as_reference_int(2 * cut) == O.ref_edge_cut(g, part, k)
            assert O.balance_ratio(g, part, k) == O.ref_balance(g, part, k)


def test_contract_clustering(graphs):
    rng = np.random.default_rng(2)
    for g in _graph_set(graphs):
        kn = O.knobs(g, 16, 0.03, 0, 0)
        for lab in (O.lp_cluster(g, kn, 0), rng.integers(0, g["n"] // 7 + 1, g["n"]).astype(np.int32)):
            c, cmap = O.contract(g, lab)
            r, rmap = O.ref_contract_clustering(g, lab)
            assert np.array_equal(cmap, rmap)
            rc = O.canonical(r)
            for key in ("xadj", "adjncy", "adjwgt", "vwgt"):
                assert np.array_equal(c[key], rc[key]), key


def test_contract_matching(graphs):
    for g in _graph_set(graphs):
        # a greedy matching along the adjacency order
        match = np.arange(g["n"], dtype=np.int32)
        used = np.zeros(g["n"], bool)
        for v in range(g["n"]):
            if used[v]:
                continue
            for e in range(g["xadj"][v], g["xadj"][v + 1]):
                u = g["adjncy"][e]
                if u != v and not used[u]:
                    match[v], match[u] = u, v
                    used[u] = used[v] = True
                    break
            used[v] = True
        label = np.minimum(np.arange(g["n"]), match).astype(np.int32)
        c, cmap = O.contract(g, label)
        r, rmap = O.ref_contract_matching(g, match)
        assert np.array_equal(cmap, rmap)
        rc = O.canonical(r)
        for key in ("xadj", "adjncy", "adjwgt", "vwgt"):
            assert np.array_equal(c[key], rc[key]), key


@pytest.mark.parametrize("bound,rounds", [(40, 1), (40, 10), (200, 10), (5000, 3)])
def test_lp_clustering_rule_matches_reference_sequential(graphs, bound, rounds):
    """size_constraint_label_propagation.cpp:134-194 on tie-free inputs, in the
    reference's own node order: the oracle's rule must reproduce it exactly."""
    for seed in (4, 5):
        g = tie_free(graphs.rgg2d(2000, seed=seed), seed=seed)
        order = O.ref_degree_order(g)
        ref = O.ref_lp_cluster(g, bound, rounds)
        ours = O.lp_cluster_seq(g, bound, rounds, order)
        assert np.array_equal(ref, ours)


@pytest.mark.parametrize("k,rounds", [(2, 25), (8, 5), (32, 25)])
def test_lp_refinement_rule_matches_reference_sequential(graphs, k, rounds):
    """label_propagation_refinement.cpp:21-98 (queue semantics) on tie-free inputs."""
    g = tie_free(graphs.rgg2d(3000, seed=6), seed=6)
    rng = np.random.default_rng(k)
    cuts = np.sort(rng.integers(0, g["n"], k - 1))
    part = np.searchsorted(cuts, np.arange(g["n"]), side="right").astype(np.int32)
    order = O.ref_degree_order(g)
    for bound in (int(1.03 * np.ceil(g["n"] / k)), int(1.2 * np.ceil(g["n"] / k))):
        ref = O.ref_lp_refine(g, k, bound, rounds, part)
        ours = O.lp_refine_seq(g, k, bound, rounds, order, part)
        assert np.array_equal(ref, ours)


def test_reference_example_graph_cut():
    """misc/example_library_call/interface_test.cpp:18-45: the 5-node graph, ECO, k=2."""
    g = csr_from_edges(5, [(0, 1), (0, 4), (1, 2), (1, 4), (2, 3), (3, 4)])
    cut, part = O.ref_kaffpa(g, 2, 0.03, 0, 1)
    assert cut == 2
    ours, opart, _ = O.kaffpa(g, 2, 0.03, 0, 1)
    assert ours == O.edge_cut(g, opart)
    assert ours >= 2  # 2 is optimal for this graph
