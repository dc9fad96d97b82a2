"""Heavy-edge matching of the oracle (the schedule the GPU follows): a valid
matching under the weight bound, and -- run to convergence -- exactly the
greedy matching in decreasing edge-key order, checked by a plain Python
restatement.  CPU only."""
import struct

import numpy as np
import pytest

from conftest import csr_from_edges, tie_free

from oracle import oracle as O


def _keys(g, kn, level, rating=None):
    ks = O.stream(kn.seed, 11, level, 0)
    out = {}
    for v in range(g["n"]):
        for e in range(g["xadj"][v], g["xadj"][v + 1]):
            u = int(g["adjncy"][e])
            if u <= v:
                continue
            if rating is not None:
                k1 = int(rating[e])
            else:
                w = int(g["adjwgt"][e])
                den = (int(g["vwgt"][v]) * int(g["vwgt"][u])) & 0xFFFFFFFF
                r = (1.0 * w * w / den) if den else (float("inf") if w else 0.0)
                k1 = struct.unpack("<Q", struct.pack("<d", r))[0]
            h = O.hash32(ks, O.hash32(ks, v) ^ u)
            k2 = (h << 32) | ((~(v + u)) & 0xFFFFFFFF)
            out[(v, u)] = (k1, k2)
    return out


def _greedy(g, kn, level, rating=None):
    keys = _keys(g, kn, level, rating)
    mate = [-1] * g["n"]
    for (v, u), _ in sorted(keys.items(), key=lambda kv: kv[1], reverse=True):
        if mate[v] < 0 and mate[u] < 0 and int(g["vwgt"][v]) + int(g["vwgt"][u]) <= kn.max_vertex_weight:
            mate[v], mate[u] = u, v
    return np.array([min(v, m) if m >= 0 else v for v, m in enumerate(mate)], np.int32)


def _check_valid(g, kn, lab):
    n = g["n"]
    members = {}
    for v in range(n):
        assert lab[v] <= v
        members.setdefault(int(lab[v]), []).append(v)
    for leader, ms in members.items():
        assert len(ms) <= 2 and ms[0] == leader
        if len(ms) == 2:
            a, b = ms
            assert b in set(g["adjncy"][g["xadj"][a]:g["xadj"][a + 1]].tolist())
            assert int(g["vwgt"][a]) + int(g["vwgt"][b]) <= kn.max_vertex_weight


@pytest.mark.parametrize("which", ["rgg2d", "rgg3d", "rmat", "tiefree", "nodew"])
def test_matching_is_greedy_order(graphs, which):
    g = {"rgg2d": lambda: graphs.rgg2d(1500, seed=1), "rgg3d": lambda: graphs.rgg3d(1200, seed=2),
         "rmat": lambda: graphs.rmat(10, seed=3), "tiefree": lambda: tie_free(graphs.rgg2d(1000, seed=4)),
         "nodew": lambda: graphs.rgg2d(1000, seed=6)}[which]()
    if which == "nodew":
        g["vwgt"] = np.random.default_rng(0).integers(1, 40, g["n"]).astype(np.int32)
    kn = O.knobs(g, 8, 0.03, 3, 0)
    if which == "nodew":
        kn.max_vertex_weight = 45  # make the weight bound bite
    kn.match_rounds = 1000
    lab = O.hem_match(g, kn, 2)
    _check_valid(g, kn, lab)
    assert np.array_equal(lab, _greedy(g, kn, 2))


def test_matching_with_supplied_rating(graphs):
    g = graphs.rgg2d(800, seed=9)
    src = np.repeat(np.arange(g["n"]), np.diff(g["xadj"]))
    rating = ((np.minimum(src, g["adjncy"]) * 2654435761 + np.maximum(src, g["adjncy"])) % 97).astype(np.uint32)
    kn = O.knobs(g, 4, 0.03, 0, 0)
    kn.match_rounds = 1000
    lab = O.hem_match(g, kn, 0, rating)
    _check_valid(g, kn, lab)
    assert np.array_equal(lab, _greedy(g, kn, 0, rating))


def test_matching_edge_cases():
    # empty graph, isolated nodes, a single edge, weight bound excluding every pair
    g = csr_from_edges(5, [(1, 2)])
    kn = O.knobs(g, 2, 0.03, 0, 0)
    assert kn.max_vertex_weight == 0  # 1.5 * W / num_stop truncates to 0 on a tiny graph
    assert O.hem_match(g, kn, 0).tolist() == [0, 1, 2, 3, 4]
    kn.max_vertex_weight = 2
    assert O.hem_match(g, kn, 0).tolist() == [0, 1, 1, 3, 4]
    kn.max_vertex_weight = 1
    assert O.hem_match(g, kn, 0).tolist() == [0, 1, 2, 3, 4]
    g0 = csr_from_edges(0, [])
    assert len(O.hem_match(g0, O.knobs(g0, 2, 0.03, 0, 0), 0)) == 0


def test_matching_coarsening_quality(graphs):
    """Matching-coarsened kaffpa stays within 25% of the LP-coarsened cut."""
    g = graphs.rgg2d(1 << 15, seed=0)
    kn = O.knobs(g, 16, 0.03, 0, 0)
    cut_lp, _, st = O.kaffpa_knobs(g, kn)
    kn.coarsening = 1
    cut_m, part, st_m = O.kaffpa_knobs(g, kn)
    assert st_m.balanced and st_m.levels > st.levels
    assert cut_m <= 1.25 * cut_lp


def test_matching_gives_way_to_lp_on_stars(graphs):
    """A star cannot be matched down (one pair per hub); such a level is
    clustered by LP instead, so coarsening keeps going."""
    from conftest import csr_from_edges
    hubs, leaves = 40, 400
    edges = [(h, hubs + h * leaves + i) for h in range(hubs) for i in range(leaves)]
    edges += [(h, (h + 1) % hubs) for h in range(hubs)]
    g = csr_from_edges(hubs * (leaves + 1), edges)
    kn = O.knobs(g, 4, 0.03, 0, 0)
    kn.coarsening = 1
    kn.match_rounds = 1000
    lab = O.hem_match(g, kn, 0)
    assert len(np.unique(lab)) > 0.75 * g["n"]  # the matching alone barely shrinks it
    cut, part, st = O.kaffpa_knobs(g, kn)
    # the level was clustered by LP, which shrinks it further than the matching
    assert st.levels >= 2 and st.level_n[1] < len(np.unique(lab)) - hubs
    assert st.balanced
