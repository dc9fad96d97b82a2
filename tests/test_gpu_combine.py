"""KaFFPaE combine on the device against the oracle, bit for bit (cut and
partition), through the C ABI (kb200_kaffpa_combine)."""
import numpy as np
import pytest

from conftest import tie_free

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def N():
    from kahip_b200 import native
    assert native.device_count() > 0, "no CUDA device: the combine tests need one"
    return native


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    return oracle


@pytest.mark.parametrize("which", ["rgg2d", "rgg3d", "rmat", "tiefree", "grid"])
@pytest.mark.parametrize("mode,coarsening,k", [(0, 0, 8), (0, 1, 16), (1, 1, 8), (1, 0, 33)])
def test_combine_matches_oracle(N, O, graphs, which, mode, coarsening, k):
    g = {"rgg2d": lambda: graphs.rgg2d(1 << 14, seed=1), "rgg3d": lambda: graphs.rgg3d(1 << 13, seed=2),
         "rmat": lambda: graphs.rmat(12, seed=3), "tiefree": lambda: tie_free(graphs.rgg2d(6000, seed=4)),
         "grid": lambda: graphs.grid2d(90, 80)}[which]()
    par = []
    for seed in (21, 22):
        kn = O.knobs(g, k, 0.03, seed, mode)
        kn.coarsening = coarsening
        par.append(O.kaffpa_knobs(g, kn)[1])
    kn_o = O.knobs(g, k, 0.03, 5, mode)
    kn_o.coarsening = coarsening
    kn_d = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, 5, mode)
    kn_d.coarsening = coarsening
    cut_o, part_o, st_o = O.kaffpa_combine(g, kn_o, par[0], par[1])
    st = N.Stats()
    _, cut_d, part_d = N.kaffpa_combine(g, kn_d, par[0], par[1], stats=st)
    assert cut_d == cut_o
    assert np.array_equal(part_d, part_o)
    assert st.initial_cut == st_o.initial_cut


def test_combine_unit_weights_and_errors(N, O, graphs):
    g = graphs.rgg2d(1 << 13, seed=7)
    kn = N.derive_knobs(g["n"], None, 8, 0.03, 0, 0)
    pa = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn)[2]
    kn.seed = 1
    pb = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn)[2]
    kn_o = O.knobs(g, 8, 0.03, 1, 0)
    cut_o, part_o, _ = O.kaffpa_combine(g, kn_o, pa, pb, unit_weights=True)
    _, cut_d, part_d = N.kaffpa_combine(g, kn, pa, pb, unit_weights=True)
    assert cut_d == cut_o and np.array_equal(part_d, part_o)
    bad = pb.copy()
    bad[3] = 8
    with pytest.raises(N.KaHIPError):
        N.kaffpa_combine(g, kn, pa, bad)


@pytest.mark.parametrize("which,mode,k", [("rgg2d", 0, 8), ("rgg3d", 1, 16), ("rmat", 0, 4)])
def test_evolution_matches_oracle(N, O, graphs, which, mode, k):
    g = {"rgg2d": lambda: graphs.rgg2d(1 << 13, seed=5), "rgg3d": lambda: graphs.rgg3d(1 << 12, seed=6),
         "rmat": lambda: graphs.rmat(11, seed=7)}[which]()
    kn_o = O.knobs(g, k, 0.03, 2, mode)
    kn_d = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, 2, mode)
    cut_o, part_o, hist_o = O.kaffpae(g, kn_o, 4, 3, 2)
    _, cut_d, part_d, hist_d = N.kaffpae(g, kn_d, 4, 3, 2)
    assert cut_d == cut_o and np.array_equal(part_d, part_o)
    assert np.array_equal(hist_d, hist_o)


def test_evolution_does_not_depend_on_workers(N, graphs):
    g = graphs.rgg2d(1 << 13, seed=8)
    kn = N.derive_knobs(g["n"], g["vwgt"], 8, 0.03, 3, 0)
    runs = [N.kaffpae(g, kn, 5, 2, 3, workers=w) for w in (1, 2, 3)]
    for r in runs[1:]:
        assert r[1] == runs[0][1] and np.array_equal(r[2], runs[0][2]) and np.array_equal(r[3], runs[0][3])


@pytest.mark.parametrize("gname", ["empty", "single", "isolated", "star", "two_components", "big_star"])
@pytest.mark.parametrize("k", [2, 8, 100])
def test_combine_edge_cases(N, O, gname, k):
    from conftest import csr_from_edges
    from test_gpu_parity import EDGE_GRAPHS
    n, edges = EDGE_GRAPHS[gname]
    g = csr_from_edges(n, edges)
    pa = O.kaffpa(g, k, 0.03, 1, 0)[1]
    pb = O.kaffpa(g, k, 0.03, 2, 1)[1]
    kn_o = O.knobs(g, k, 0.03, 3, 0)
    kn_d = N.derive_knobs(g["n"], g["vwgt"], k, 0.03, 3, 0)
    cut_o, part_o, _ = O.kaffpa_combine(g, kn_o, pa, pb)
    _, cut_d, part_d = N.kaffpa_combine(g, kn_d, pa, pb)
    assert cut_d == cut_o and np.array_equal(part_d, part_o)
