"""Batched form: many independent graphs, and a population of seeds of one
device-resident graph.  Every member must equal the oracle's run with the
same arguments (bit-exact partition and cut)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def N():
    from kahip_b200 import native
    assert native.device_count() > 0, "no CUDA device: the GPU batch tests need one"
    return native


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    return oracle


def test_batch_mixed_graphs_match_single_runs(N, O, graphs):
    mix = graphs.batch_mix(24, seed=5, nmin=300, nmax=20000)
    gs = [g for g, _ in mix]
    ks = [k for _, k in mix]
    seeds = list(range(len(gs)))
    modes = [i % 2 for i in range(len(gs))]
    cuts, parts, status, rep = N.kaffpa_batch(gs, ks, 0.03, seeds, modes, workers=6)
    assert rep.failed == 0 and rep.workers == 6
    for g, k, s, md, c, p, stt in zip(gs, ks, seeds, modes, cuts, parts, status):
        cut_o, part_o, st_o = O.kaffpa(g, k, 0.03, s, md)
        assert stt >= 0
        assert c == cut_o
        assert np.array_equal(p, part_o)
    # one worker gives the same results
    cuts1, parts1, _, rep1 = N.kaffpa_batch(gs, ks, 0.03, seeds, modes, workers=1)
    assert rep1.workers == 1
    assert np.array_equal(cuts1, cuts)
    assert all(np.array_equal(a, b) for a, b in zip(parts, parts1))


def test_batch_reports_bad_items(N, graphs):
    good = graphs.rgg2d(2000, seed=1)
    bad = dict(good)
    bad["adjncy"] = good["adjncy"].copy()
    bad["adjncy"][5] = good["n"] + 7  # target out of range
    cuts, parts, status, rep = N.kaffpa_batch([good, bad, good], [4, 4, 8], 0.03, 0, 0, workers=2)
    assert rep.failed == 1
    assert status[0] >= 0 and status[2] >= 0 and status[1] == -1
    assert cuts[1] == -1 and cuts[0] > 0 and cuts[2] > 0


def test_population_of_seeds(N, O, graphs):
    import torch
    g = graphs.rgg2d(1 << 14, seed=3)
    dev = torch.device("cuda:0")
    n = g["n"]
    t = {k: torch.from_numpy(np.ascontiguousarray(g[k], np.int32)).to(dev) for k in ("xadj", "adjncy", "adjwgt", "vwgt")}
    seeds = [0, 1, 2, 3, 17, 100, 1000, 12345]
    parts = torch.empty(len(seeds) * n, dtype=torch.int32, device=dev)
    cuts, rep = N.kaffpa_population(n, t["xadj"], t["adjncy"], t["adjwgt"], t["vwgt"], parts, 16, seeds,
                                    workers=4)
    assert rep.failed == 0
    host = parts.cpu().numpy().reshape(len(seeds), n)
    for i, s in enumerate(seeds):
        cut_o, part_o, _ = O.kaffpa(g, 16, 0.03, s, 0)
        assert cuts[i] == cut_o
        assert np.array_equal(host[i], part_o)
