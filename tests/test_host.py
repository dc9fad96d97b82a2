"""Host logic of the product against the oracle, no GPU needed: knob
derivation (bounds, stop rule, presets) and the host initial partitioner."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("n,k,imb,mode,weighted", [(1 << 24, 64, 0.03, 0, False), (1 << 15, 8, 0.03, 1, True),
                                                   (5000, 3, 0.0, 0, True), (100, 7, 0.1, 2, False),
                                                   (1 << 20, 256, 0.05, 3, False), (1, 1, 0.03, 9, False),
                                                   (0, 4, 0.03, 0, False)])
def test_knobs_match_oracle(n, k, imb, mode, weighted):
    from kahip_b200 import native
    vw = np.random.default_rng(n).integers(1, 7, n).astype(np.int32) if weighted else None
    a = native.derive_knobs(n, vw, k, imb, 5, mode).as_dict()
    b = O.knobs(dict(n=n, vwgt=vw if vw is not None else np.ones(n, np.int32)), k, imb, 5, mode)
    assert a == {f: getattr(b, f) for f, _ in b._fields_}


@pytest.mark.parametrize("gen,k,mode,seed", [("rgg2d", 8, 0, 0), ("rgg2d", 64, 0, 0), ("rgg2d", 64, 1, 5),
                                             ("rgg3d", 13, 1, 2), ("rmat", 16, 0, 1), ("grid", 2, 0, 1),
                                             ("rgg2d", 256, 0, 3)])
def test_initial_partitioner_matches_oracle(graphs, gen, k, mode, seed):
    from kahip_b200 import native
    g = {"rgg2d": lambda: graphs.rgg2d(1 << 15, seed=seed), "rgg3d": lambda: graphs.rgg3d(1 << 14, seed=seed),
         "rmat": lambda: graphs.rmat(13, seed=seed), "grid": lambda: graphs.grid2d(120, 100)}[gen]()
    kn = O.knobs(g, k, 0.03, seed, mode)
    c, _ = O.contract(g, O.lp_cluster(g, kn, 0))
    a = O.initial_partition(c, kn)
    b = native.initial_partition(c, native.derive_knobs(g["n"], g["vwgt"], k, 0.03, seed, mode))
    assert np.array_equal(a, b)
    assert a.min() >= 0 and a.max() < k


@pytest.mark.parametrize("k,mode", [(8, 0), (16, 1)])
def test_initial_partitioner_dense_graph_matches_oracle(k, mode):
    # average degree > 64: one growing try and one FM pass per bisection, in both
    from conftest import csr_from_edges
    from kahip_b200 import native
    rng = np.random.default_rng(k)
    n = 400
    edges = set()
    while len(edges) < 14000:
        u, v = rng.integers(0, n, 2)
        if u != v:
            edges.add((min(u, v), max(u, v)))
    g = csr_from_edges(n, sorted(edges), weights=list(rng.integers(1, 9, len(edges))))
    g["vwgt"] = rng.integers(1, 5, n).astype(np.int32)
    assert g["m"] > 64 * n
    kn = O.knobs(g, k, 0.03, 1, mode)
    a = O.initial_partition(g, kn)
    b = native.initial_partition(g, native.derive_knobs(g["n"], g["vwgt"], k, 0.03, 1, mode))
    assert np.array_equal(a, b)


def test_generators_are_symmetric_and_sorted(graphs):
    for g in (graphs.rgg2d(5000, seed=1), graphs.rgg3d(4000, seed=2), graphs.rmat(12, seed=3),
              graphs.grid2d(50, 40)):
        n, xadj, adj, w = g["n"], g["xadj"], g["adjncy"], g["adjwgt"]
        src = np.repeat(np.arange(n), np.diff(xadj))
        assert (adj != src).all(), "self loop"
        fwd = set(zip(src.tolist(), adj.tolist(), w.tolist()))
        rev = set(zip(adj.tolist(), src.tolist(), w.tolist()))
        assert fwd == rev, "not symmetric"
        for v in range(0, n, max(1, n // 200)):
            row = adj[xadj[v]:xadj[v + 1]]
            assert (np.diff(row) > 0).all(), "row not sorted / duplicate"


def test_rgg_average_degree_matches_spec(graphs):
    g = graphs.rgg2d(1 << 16, seed=0)
    # 2D RGG with r = 0.55 sqrt(ln n / n): expected average degree ~ 0.95 ln n
    assert abs(g["m"] / g["n"] - 0.95 * np.log(g["n"])) < 0.6
