"""CUDA path vs the CPU oracle, phase by phase and end to end, bit-exact.

Every test here calls the product through its C ABI (libkahip_b200.so via
kahip_b200.native) and the oracle through oracle/liboracle.so, on identical
seeded inputs.  Integer / index outputs must match exactly.
"""
import numpy as np
import pytest

from conftest import csr_from_edges, tie_free

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def N():
    from kahip_b200 import native
    assert native.device_count() > 0, "no CUDA device: the GPU parity tests need one"
    return native


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    return oracle


def _cases(graphs):
    out = {
        "rgg2d_15": graphs.rgg2d(1 << 15, seed=0),
        "rgg2d_12_s3": graphs.rgg2d(1 << 12, seed=3),
        "rgg3d_13": graphs.rgg3d(1 << 13, seed=1),
        "grid_60x50": graphs.grid2d(60, 50),
        "rmat_12": graphs.rmat(12, seed=2),
    }
    out["rgg2d_14_weighted"] = tie_free(graphs.rgg2d(1 << 14, seed=5))
    g = graphs.rgg2d(1 << 13, seed=9)
    rng = np.random.default_rng(4)
    g["vwgt"] = rng.integers(1, 6, size=g["n"]).astype(np.int32)
    out["rgg2d_13_nodeweights"] = g
    return out


@pytest.fixture(scope="module")
def cases(graphs):
    return _cases(graphs)


CASE_NAMES = ["rgg2d_15", "rgg2d_12_s3", "rgg3d_13", "grid_60x50", "rmat_12", "rgg2d_14_weighted",
              "rgg2d_13_nodeweights"]


@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("k,mode,seed", [(8, 0, 0), (64, 1, 3)])
def test_lp_cluster_parity(N, O, cases, name, k, mode, seed):
    g = cases[name]
    kn_o = O.knobs(g, k, 0.03, seed, mode)
    kn_p = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, seed, mode)
    for level in (0, 2):
        a = O.lp_cluster(g, kn_o, level)
        b = N.lp_cluster(g, kn_p, level)
        assert np.array_equal(a, b), f"clustering differs at {np.flatnonzero(a != b)[:10]}"


@pytest.mark.parametrize("name", CASE_NAMES)
def test_contract_parity(N, O, cases, name):
    g = cases[name]
    kn = O.knobs(g, 16, 0.03, 1, 0)
    lab = O.lp_cluster(g, kn, 0)
    co, cmo = O.contract(g, lab)
    cp, cmp_ = N.contract(g, lab)
    assert np.array_equal(cmo, cmp_)
    for key in ("xadj", "adjncy", "adjwgt", "vwgt"):
        assert np.array_equal(co[key], cp[key]), key
    # arbitrary (non-LP) labels, including singleton-only and all-in-one
    rng = np.random.default_rng(0)
    for lab in (rng.integers(0, g["n"], g["n"]), np.arange(g["n"]), np.zeros(g["n"])):
        co, cmo = O.contract(g, lab)
        cp, cmp_ = N.contract(g, lab)
        assert np.array_equal(cmo, cmp_)
        for key in ("xadj", "adjncy", "adjwgt", "vwgt"):
            assert np.array_equal(co[key], cp[key]), key


@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("k", [2, 8, 64])
def test_refine_and_balance_parity(N, O, cases, name, k):
    g = cases[name]
    kn_o = O.knobs(g, k, 0.03, 2, 1)
    kn_p = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, 2, 1)
    rng = np.random.default_rng(k)
    # a spatially coherent but unbalanced start: blocks by node id ranges, skewed
    cuts = np.sort(rng.integers(0, g["n"], k - 1))
    part = np.searchsorted(cuts, np.arange(g["n"]), side="right").astype(np.int32)
    for level in (0, 1):
        pb_o, ok_o = O.balance(g, kn_o, part, kn_o.upper_bound, level)
        pb_p, ok_p = N.balance(g, kn_p, part, kn_p.upper_bound, level)
        assert ok_o == ok_p
        assert np.array_equal(pb_o, pb_p)
        pr_o = O.lp_refine(g, kn_o, pb_o, kn_o.upper_bound, level)
        pr_p = N.lp_refine(g, kn_p, pb_o, kn_p.upper_bound, level)
        assert np.array_equal(pr_o, pr_p)


@pytest.mark.parametrize("name", CASE_NAMES)
def test_edge_cut_and_block_weights(N, O, cases, name):
    g = cases[name]
    rng = np.random.default_rng(1)
    for k in (1, 2, 7, 300):
        part = rng.integers(0, k, g["n"]).astype(np.int32)
        cut, bw = N.edge_cut(g, part, k)
        assert cut == O.edge_cut(g, part)
        assert np.array_equal(bw, O.block_weights(g, part, k))


def test_project(N):
    rng = np.random.default_rng(3)
    cmap = rng.integers(0, 1000, 50000).astype(np.int32)
    pc = rng.integers(0, 16, 1000).astype(np.int32)
    assert np.array_equal(N.project(cmap, 1000, pc), pc[cmap])


@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("k,mode,seed", [(2, 0, 0), (8, 0, 1), (64, 0, 0), (16, 1, 4), (5, 1, 2)])
def test_kaffpa_end_to_end(N, O, cases, name, k, mode, seed):
    g = cases[name]
    cut_o, part_o, st_o = O.kaffpa(g, k, 0.03, seed, mode)
    st = N.Stats()
    st.collect_level_cuts = 1
    rc, cut_p, part_p = N.kaffpa_ex(g["xadj"], g["adjncy"], k, 0.03, seed, mode, vwgt=g["vwgt"],
                                    adjwgt=g["adjwgt"], stats=st)
    assert st.levels == st_o.levels
    for l in range(st.levels):
        assert st.level_n[l] == st_o.level_n[l], l
        assert st.level_m[l] == st_o.level_m[l], l
        assert st.level_cut[l] == st_o.level_cut[l], l
        assert st.level_maxbw[l] == st_o.level_maxbw[l], l
    assert st.initial_cut == st_o.initial_cut
    assert cut_p == cut_o
    assert np.array_equal(part_p, part_o)
    kn = O.knobs(g, k, 0.03, seed, mode)
    bw = O.block_weights(g, part_p, k)
    assert (rc == 0) == (bw.max() <= kn.final_bound)
    assert bw.max() <= kn.final_bound, "imbalance bound violated"


def test_drop_in_kaffpa_abi(N, O, graphs):
    """kaffpa() with the reference signature (int*/double* arguments, NULL weights)."""
    import ctypes
    g = graphs.rgg2d(1 << 12, seed=0)
    L = N.lib()
    n = ctypes.c_int(g["n"])
    k = ctypes.c_int(4)
    imb = ctypes.c_double(0.03)
    cut = ctypes.c_int(-7)
    part = np.zeros(g["n"], np.int32)
    L.kaffpa(ctypes.byref(n), None, g["xadj"].ctypes.data, None, g["adjncy"].ctypes.data, ctypes.byref(k),
             ctypes.byref(imb), True, 0, 0, ctypes.byref(cut), part.ctypes.data)
    cut_o, part_o, _ = O.kaffpa(g, 4, 0.03, 0, 0, unit_weights=True)
    assert cut.value == cut_o
    assert np.array_equal(part, part_o)


@pytest.mark.parametrize("perfectly_balance", [False, True])
def test_drop_in_kaffpa_balance_keeps_epsilon(N, O, graphs, perfectly_balance):
    """kaffpa_balance keeps the caller's epsilon for either flag value: the
    reference's perfectly_balance enforces max block <= (1+eps)*ceil(W/k)
    after partitioning (interface/kaHIP_interface.cpp:115-129), the bound
    every partition here already meets."""
    import ctypes
    g = graphs.rgg2d(1 << 12, seed=2)
    rng = np.random.default_rng(5)
    vwgt = rng.integers(1, 4, g["n"]).astype(np.int32)
    L = N.lib()
    n = ctypes.c_int(g["n"])
    k = ctypes.c_int(8)
    imb = ctypes.c_double(0.03)
    cut = ctypes.c_int(-7)
    part = np.zeros(g["n"], np.int32)
    L.kaffpa_balance(ctypes.byref(n), vwgt.ctypes.data, g["xadj"].ctypes.data, None, g["adjncy"].ctypes.data,
                     ctypes.byref(k), ctypes.byref(imb), ctypes.c_bool(perfectly_balance), True, 0, 0,
                     ctypes.byref(cut), part.ctypes.data)
    gw = dict(g, vwgt=vwgt)
    cut_o, part_o, _ = O.kaffpa(gw, 8, 0.03, 0, 0)
    assert cut.value == cut_o
    assert np.array_equal(part, part_o)
    W = int(vwgt.sum())
    bound = int((1 + 0.03) * -(-W // 8))
    assert O.block_weights(gw, part, 8).max() <= bound


@pytest.mark.parametrize("gen,k,mode,seed", [("rgg2d", 8, 0, 0), ("rgg2d", 64, 0, 0), ("rgg2d", 64, 1, 5),
                                             ("rgg3d", 13, 1, 2), ("rmat", 16, 0, 1), ("grid", 2, 0, 1),
                                             ("rgg2d", 256, 0, 3), ("grid", 7, 1, 4)])
def test_device_initial_partitioner_matches_oracle(N, O, graphs, gen, k, mode, seed):
    """The device's batched recursive bisection on a coarsest-like graph (one
    level of oracle LP clustering) against its oracle restatement."""
    g = {"rgg2d": lambda: graphs.rgg2d(1 << 15, seed=seed), "rgg3d": lambda: graphs.rgg3d(1 << 14, seed=seed),
         "rmat": lambda: graphs.rmat(13, seed=seed), "grid": lambda: graphs.grid2d(120, 100)}[gen]()
    kn = O.knobs(g, k, 0.03, seed, mode)
    c, _ = O.contract(g, O.lp_cluster(g, kn, 0))
    a = O.initial_partition_batched(c, kn)
    b = N.initial_partition_device(c, N.derive_knobs(g["n"], g["vwgt"], k, 0.03, seed, mode))
    assert np.array_equal(a, b)
    assert a.min() >= 0 and a.max() < k


@pytest.mark.parametrize("k,mode", [(8, 0), (16, 1)])
def test_device_initial_partitioner_dense_graph(N, O, k, mode):
    # average degree > 64: one try per bisection, rows walked by whole warps
    rng = np.random.default_rng(k)
    n = 400
    edges = set()
    while len(edges) < 14000:
        u, v = rng.integers(0, n, 2)
        if u != v:
            edges.add((min(u, v), max(u, v)))
    g = csr_from_edges(n, sorted(edges), weights=list(rng.integers(1, 9, len(edges))))
    g["vwgt"] = rng.integers(1, 5, n).astype(np.int32)
    kn = O.knobs(g, k, 0.03, 1, mode)
    a = O.initial_partition_batched(g, kn)
    b = N.initial_partition_device(g, N.derive_knobs(g["n"], g["vwgt"], k, 0.03, 1, mode))
    assert np.array_equal(a, b)


@pytest.mark.parametrize("gname", ["single", "isolated", "path", "star", "two_components"])
@pytest.mark.parametrize("k", [2, 3, 8, 100])
def test_device_initial_partitioner_edge_cases(N, O, gname, k):
    n, edges = EDGE_GRAPHS[gname]
    g = csr_from_edges(n, edges)
    kn = O.knobs(g, k, 0.03, 0, 0)
    a = O.initial_partition_batched(g, kn)
    b = N.initial_partition_device(g, N.derive_knobs(g["n"], g["vwgt"], k, 0.03, 0, 0))
    assert np.array_equal(a, b)


EDGE_GRAPHS = {
    "empty": (0, []),
    "single": (1, []),
    "isolated": (50, []),
    "path": (40, [(i, i + 1) for i in range(39)]),
    "star": (65, [(0, i) for i in range(1, 65)]),
    "clique": (24, [(i, j) for i in range(24) for j in range(i + 1, 24)]),
    "two_components": (60, [(i, i + 1) for i in range(29)] + [(i, i + 1) for i in range(30, 59)]),
    "big_star": (3000, [(0, i) for i in range(1, 3000)] + [(i, i + 1) for i in range(1, 2999)]),
}


@pytest.mark.parametrize("gname", list(EDGE_GRAPHS))
@pytest.mark.parametrize("k", [1, 2, 3, 8, 100])
@pytest.mark.parametrize("mode", [0, 1])
def test_edge_cases(N, O, gname, k, mode):
    n, edges = EDGE_GRAPHS[gname]
    g = csr_from_edges(n, edges)
    cut_o, part_o, st_o = O.kaffpa(g, k, 0.03, 0, mode)
    rc, cut_p, part_p = N.kaffpa_ex(g["xadj"], g["adjncy"], k, 0.03, 0, mode)
    assert cut_p == cut_o
    assert np.array_equal(part_p, part_o)
    if n:
        assert part_p.min() >= 0 and part_p.max() < k


def test_imbalance_zero_and_weighted_nodes(N, O, graphs):
    g = graphs.rgg2d(1 << 12, seed=11)
    rng = np.random.default_rng(5)
    g["vwgt"] = rng.integers(1, 4, g["n"]).astype(np.int32)
    for imb in (0.0, 0.01, 0.1):
        cut_o, part_o, _ = O.kaffpa(g, 6, imb, 0, 0)
        rc, cut_p, part_p = N.kaffpa_ex(g["xadj"], g["adjncy"], 6, imb, 0, 0, vwgt=g["vwgt"], adjwgt=g["adjwgt"])
        assert cut_p == cut_o
        assert np.array_equal(part_p, part_o)


def test_invalid_input_rejected(N):
    from kahip_b200.native import KaHIPError
    with pytest.raises(KaHIPError):
        N.kaffpa_ex(np.array([0, 2, 1]), np.array([1, 0]), 2)       # xadj not monotone
    with pytest.raises(KaHIPError):
        N.kaffpa_ex(np.array([0, 1, 2]), np.array([1, 5]), 2)       # target out of range
    with pytest.raises(KaHIPError):
        N.kaffpa_ex(np.array([0, 1, 2]), np.array([1, 0]), 0)       # k < 1


def _sym_rating(g, seed):
    """A symmetric uint32 rating per directed entry (stands in for a learned one)."""
    rng = np.random.default_rng(seed)
    n, xadj, adj = g["n"], g["xadj"], g["adjncy"]
    src = np.repeat(np.arange(n), np.diff(xadj))
    key = np.minimum(src, adj).astype(np.int64) * n + np.maximum(src, adj)
    uniq, inv = np.unique(key, return_inverse=True)
    r = rng.integers(0, 1 << 12, size=len(uniq)).astype(np.uint32)  # many equal ratings
    return r[inv]


@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("k,seed", [(8, 0), (64, 5)])
def test_hem_match_parity(N, O, cases, name, k, seed):
    g = cases[name]
    kn_o = O.knobs(g, k, 0.03, seed, 0)
    kn_p = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, seed, 0)
    for level in (0, 3):
        a = O.hem_match(g, kn_o, level)
        b = N.hem_match(g, kn_p, level)
        assert np.array_equal(a, b), f"matching differs at {np.flatnonzero(a != b)[:10]}"
    rq = _sym_rating(g, seed)
    a = O.hem_match(g, kn_o, 1, rq)
    b = N.hem_match(g, kn_p, 1, rq)
    assert np.array_equal(a, b)
    # a capped number of rounds is part of the schedule too
    kn_o.match_rounds = kn_p.match_rounds = 2
    assert np.array_equal(O.hem_match(g, kn_o, 0), N.hem_match(g, kn_p, 0))


@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("k,mode,seed", [(8, 0, 0), (64, 1, 2)])
def test_kaffpa_matching_coarsening_parity(N, O, cases, name, k, mode, seed):
    g = cases[name]
    kn_o = O.knobs(g, k, 0.03, seed, mode)
    kn_p = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, seed, mode)
    kn_o.coarsening = kn_p.coarsening = 1
    cut_o, part_o, st_o = O.kaffpa_knobs(g, kn_o)
    st = N.Stats()
    st.collect_level_cuts = 1
    rc, cut_p, part_p = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn_p, vwgt=g["vwgt"], adjwgt=g["adjwgt"], stats=st)
    assert st.levels == st_o.levels
    for l in range(st.levels):
        assert (st.level_n[l], st.level_m[l], st.level_cut[l], st.level_maxbw[l]) == \
               (st_o.level_n[l], st_o.level_m[l], st_o.level_cut[l], st_o.level_maxbw[l]), l
    assert cut_p == cut_o
    assert np.array_equal(part_p, part_o)
    assert O.block_weights(g, part_p, k).max() <= kn_o.final_bound


def test_matching_hub_rows(N, O):
    """Rows longer than a warp's lane budget take the warp-cooperative path."""
    n = 3000
    edges = [(0, v) for v in range(1, n)] + [(v, v + 1) for v in range(1, n - 1)] + \
            [(7, v) for v in range(100, 900)]
    g = csr_from_edges(n, edges, weights=[1 + (i * 7919) % 13 for i in range(len(edges))])
    for k in (2, 16):
        kn_o = O.knobs(g, k, 0.03, 1, 0)
        kn_p = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, 1, 0)
        assert np.array_equal(O.hem_match(g, kn_o, 0), N.hem_match(g, kn_p, 0))


@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("k,level", [(8, 0), (33, 2)])
def test_jet_refine_parity(N, O, cases, name, k, level):
    g = cases[name]
    kn_o = O.knobs(g, k, 0.03, 3, 1)
    kn_p = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, 3, 1)
    rng = np.random.default_rng(k)
    part = (np.arange(g["n"]) * k // g["n"]).astype(np.int32)
    flip = rng.random(g["n"]) < 0.05
    part[flip] = rng.integers(0, k, flip.sum())
    a = O.jet_refine(g, kn_o, part, kn_o.upper_bound, level)
    b = N.jet_refine(g, kn_p, part, kn_p.upper_bound, level)
    assert np.array_equal(a, b), f"Jet differs at {np.flatnonzero(a != b)[:10]}"


@pytest.mark.parametrize("name", CASE_NAMES)
@pytest.mark.parametrize("k,mode,seed", [(8, 0, 0), (64, 1, 2)])
def test_kaffpa_jet_parity(N, O, cases, name, k, mode, seed):
    g = cases[name]
    kn_o = O.knobs(g, k, 0.03, seed, mode)
    kn_p = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, seed, mode)
    kn_o.refinement = kn_p.refinement = 1
    cut_o, part_o, st_o = O.kaffpa_knobs(g, kn_o)
    st = N.Stats()
    st.collect_level_cuts = 1
    rc, cut_p, part_p = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn_p, vwgt=g["vwgt"], adjwgt=g["adjwgt"], stats=st)
    assert st.levels == st_o.levels
    for l in range(st.levels):
        assert (st.level_cut[l], st.level_maxbw[l]) == (st_o.level_cut[l], st_o.level_maxbw[l]), l
    assert cut_p == cut_o and np.array_equal(part_p, part_o)
    assert O.block_weights(g, part_p, k).max() <= kn_o.final_bound


def test_jet_hub_rows(N, O):
    """Rows past the lane path's limits (many distinct blocks, long rows)."""
    n = 5000
    edges = [(0, v) for v in range(1, n)] + [(v, v + 1) for v in range(1, n - 1)] + \
            [(1, v) for v in range(2000, 2600)]
    g = csr_from_edges(n, edges, weights=[1 + (i * 13) % 7 for i in range(len(edges))])
    for k in (16, 100):
        kn_o = O.knobs(g, k, 0.05, 1, 1)
        kn_p = N.derive_knobs(g["n"], g["vwgt"], k, 0.05, 1, 1)
        part = (np.arange(n) * k // n).astype(np.int32)
        assert np.array_equal(O.jet_refine(g, kn_o, part, kn_o.upper_bound, 1),
                              N.jet_refine(g, kn_p, part, kn_p.upper_bound, 1))


@pytest.mark.parametrize("mode", [0, 1])
def test_unsorted_rows_with_parallel_entries(N, O, graphs, mode):
    # rows in arbitrary order, some edges listed twice (both directions): the
    # device check must see that rows are not strictly increasing, so that
    # clustering round 0 aggregates repeated targets like the oracle
    g = graphs.rgg2d(1 << 13, seed=3)
    rng = np.random.default_rng(1)
    n = g["n"]
    src = np.repeat(np.arange(n), np.diff(g["xadj"]))
    dst = g["adjncy"]
    upper = src < dst
    us, vs = src[upper], dst[upper]
    dup = rng.random(len(us)) < 0.15
    us = np.concatenate([us, us[dup]])
    vs = np.concatenate([vs, vs[dup]])
    ws = rng.integers(1, 5, len(us))
    a = np.concatenate([us, vs])
    b = np.concatenate([vs, us])
    w = np.concatenate([ws, ws])
    order = np.lexsort((rng.random(len(a)), a))  # by source, random within a row
    a, b, w = a[order], b[order], w[order]
    xadj = np.concatenate([[0], np.cumsum(np.bincount(a, minlength=n))]).astype(np.int32)
    h = {"n": n, "m": len(a), "xadj": xadj, "adjncy": b.astype(np.int32), "adjwgt": w.astype(np.int32),
         "vwgt": np.ones(n, np.int32)}
    cut_o, part_o, _ = O.kaffpa(h, 8, 0.03, 0, mode)
    rc, cut_p, part_p = N.kaffpa_ex(h["xadj"], h["adjncy"], 8, 0.03, 0, mode, vwgt=h["vwgt"], adjwgt=h["adjwgt"])
    assert cut_p == cut_o
    assert np.array_equal(part_p, part_o)
