"""KaFFPaE combine in the oracle (CPU): the coarsest graph keeps every cut
edge of the better parent (its initial cut equals that parent's cut), the
child is never worse than the better parent by (overload, cut), the better
parent is chosen whatever the argument order, and the result is
deterministic."""
import numpy as np
import pytest

from conftest import tie_free

from oracle import oracle as O


def parents(g, k, mode, coarsening):
    out = []
    for seed in (11, 12):
        kn = O.knobs(g, k, 0.03, seed, mode)
        kn.coarsening = coarsening
        out.append(O.kaffpa_knobs(g, kn)[1])
    return out


def quality(g, part, k, bound):
    bw = O.block_weights(g, part, k)
    return int(np.maximum(bw.astype(np.int64) - bound, 0).sum()), O.edge_cut(g, part)


@pytest.mark.parametrize("which", ["rgg2d", "rgg3d", "rmat", "tiefree"])
@pytest.mark.parametrize("mode,coarsening", [(0, 0), (0, 1), (1, 1)])
def test_child_keeps_parent_cut_edges_and_never_worsens(graphs, which, mode, coarsening):
    g = {"rgg2d": lambda: graphs.rgg2d(1 << 13, seed=1), "rgg3d": lambda: graphs.rgg3d(1 << 12, seed=2),
         "rmat": lambda: graphs.rmat(11, seed=3), "tiefree": lambda: tie_free(graphs.rgg2d(5000, seed=4))}[which]()
    k = 8
    pa, pb = parents(g, k, mode, coarsening)
    kn = O.knobs(g, k, 0.03, 3, mode)
    kn.coarsening = coarsening
    qa, qb = quality(g, pa, k, kn.final_bound), quality(g, pb, k, kn.final_bound)
    better = pa if qa <= qb else pb
    cut, part, st = O.kaffpa_combine(g, kn, pa, pb)
    assert st.initial_cut == O.edge_cut(g, better)
    q = quality(g, part, k, kn.final_bound)
    assert q <= min(qa, qb) and cut == q[1]
    if qa != qb:
        cut2, part2, _ = O.kaffpa_combine(g, kn, pb, pa)
        assert cut2 == cut and np.array_equal(part2, part)
    assert np.array_equal(O.kaffpa_combine(g, kn, pa, pb)[1], part)


def test_identical_parents_and_empty_graph(graphs):
    g = graphs.rgg2d(3000, seed=9)
    kn = O.knobs(g, 4, 0.03, 0, 0)
    p = O.kaffpa_knobs(g, kn)[1]
    cut, part, st = O.kaffpa_combine(g, kn, p, p)
    assert st.initial_cut == O.edge_cut(g, p) and cut <= O.edge_cut(g, p)
    e = {"n": 0, "m": 0, "xadj": np.zeros(1, np.int32), "adjncy": np.zeros(0, np.int32),
         "adjwgt": np.zeros(0, np.int32), "vwgt": np.zeros(0, np.int32)}
    cut, part, _ = O.kaffpa_combine(e, O.knobs(e, 4, 0.03, 0, 0), np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert cut == 0 and len(part) == 0


def test_rejects_out_of_range_parent(graphs):
    g = graphs.rgg2d(500, seed=1)
    kn = O.knobs(g, 4, 0.03, 0, 0)
    p = np.zeros(g["n"], np.int32)
    q = p.copy()
    q[7] = 4
    with pytest.raises(ValueError):
        O.kaffpa_combine(g, kn, p, q)


@pytest.mark.parametrize("mode", [0, 1])
def test_evolution_never_loses_its_best(graphs, mode):
    g = graphs.rgg2d(1 << 12, seed=2)
    kn = O.knobs(g, 8, 0.03, 4, mode)
    cut, part, hist = O.kaffpae(g, kn, 4, 3, 2)
    assert all(hist[i + 1] <= hist[i] for i in range(len(hist) - 1))
    assert cut == hist[-1] == O.edge_cut(g, part)
    # the initial population is the plain partitioner with seeds seed + i
    firsts = []
    for i in range(4):
        k2 = O.knobs(g, 8, 0.03, 4 + i, mode)
        firsts.append(O.kaffpa_knobs(g, k2)[0])
    assert hist[0] == min(firsts)
    again = O.kaffpae(g, kn, 4, 3, 2)
    assert again[0] == cut and np.array_equal(again[1], part)


def test_evolution_single_member_is_the_plain_partitioner(graphs):
    g = graphs.rgg2d(2000, seed=3)
    kn = O.knobs(g, 4, 0.03, 9, 0)
    cut, part, hist = O.kaffpae(g, kn, 1, 2, 1)
    c0, p0, _ = O.kaffpa_knobs(g, kn)
    assert cut == c0 and np.array_equal(part, p0) and list(hist) == [c0] * 3


def _evolve_restated(g, kn_base, P, G, W):
    """The evolution loop restated in Python on top of the oracle's kaffpa and
    combine (tournament of two hash-drawn members twice, offspring inserted in
    order: dropped when worse than the worst member, else replacing the most
    similar member among those not better), an independent check of
    or_kaffpae's bookkeeping."""
    n = g["n"]
    src = np.repeat(np.arange(n), np.diff(g["xadj"]))
    dst = g["adjncy"]
    k = kn_base.k

    def obj(p):
        bw = O.block_weights(g, p, k).astype(np.int64)
        return (int(np.maximum(bw - kn_base.final_bound, 0).sum()), O.edge_cut(g, p))

    def fitter(objs, a, b):
        if objs[a] < objs[b]:
            return a
        if objs[b] < objs[a]:
            return b
        return min(a, b)

    pop, objs = [], []
    for i in range(P):
        kn = type(kn_base).from_buffer_copy(kn_base)
        kn.seed = kn_base.seed + i
        p = O.kaffpa_knobs(g, kn)[1]
        pop.append(p)
        objs.append(obj(p))
    best = 0
    for i in range(1, P):
        best = fitter(objs, best, i)
    hist = [objs[best][1]]
    for t in range(G):
        if P >= 2:
            offs = []
            for j in range(W):
                ks = O.stream(kn_base.seed, 13, t, j)
                x = [(O.hash32(ks, i) * P) >> 32 for i in range(4)]  # multiply-shift range
                a = fitter(objs, x[0], x[1])
                b = fitter(objs, x[2], x[3])
                if b == a:
                    b = x[3] if b == x[2] else x[2]
                if b == a:
                    b = (a + 1) % P
                kn = type(kn_base).from_buffer_copy(kn_base)
                kn.seed = kn_base.seed + P + t * W + j
                child = O.kaffpa_combine(g, kn, pop[a], pop[b])[1]
                offs.append((child, obj(child)))
            for child, oc in offs:
                worst = 0
                for i in range(1, P):
                    if objs[worst] < objs[i]:
                        worst = i
                if objs[worst] < oc:
                    continue
                pick, pd = -1, 0
                for i in range(P):
                    if objs[i] < oc:
                        continue
                    d = int(((pop[i][src] != pop[i][dst]) != (child[src] != child[dst])).sum())
                    if pick < 0 or d < pd:
                        pick, pd = i, d
                pop[pick] = child
                objs[pick] = oc
        best = 0
        for i in range(1, P):
            best = fitter(objs, best, i)
        hist.append(objs[best][1])
    return pop[best], hist


@pytest.mark.parametrize("mode", [0, 1])
def test_evolution_matches_python_restatement(graphs, mode):
    g = graphs.rgg2d(3000, seed=5)
    kn = O.knobs(g, 4, 0.03, 7, mode)
    cut, part, hist = O.kaffpae(g, kn, 4, 3, 2)
    p2, h2 = _evolve_restated(g, kn, 4, 3, 2)
    assert list(hist) == h2
    assert np.array_equal(part, p2)
