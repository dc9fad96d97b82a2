"""Jet refinement in the oracle (CPU): it keeps the bound, never returns a
worse partition than it was given (by overload, then cut), and improves on
LP refinement end to end."""
import numpy as np
import pytest

from conftest import tie_free

from oracle import oracle as O


def start_partition(g, k, seed):
    rng = np.random.default_rng(seed)
    # blocks of consecutive ids (spatially coherent for the sorted generators) plus noise
    part = (np.arange(g["n"]) * k // g["n"]).astype(np.int32)
    flip = rng.random(g["n"]) < 0.05
    part[flip] = rng.integers(0, k, flip.sum())
    return part


@pytest.mark.parametrize("which", ["rgg2d", "rgg3d", "grid", "rmat", "tiefree"])
def test_jet_keeps_bound_and_never_worsens(graphs, which):
    g = {"rgg2d": lambda: graphs.rgg2d(1 << 13, seed=1), "rgg3d": lambda: graphs.rgg3d(1 << 12, seed=2),
         "grid": lambda: graphs.grid2d(70, 60), "rmat": lambda: graphs.rmat(11, seed=3),
         "tiefree": lambda: tie_free(graphs.rgg2d(5000, seed=4))}[which]()
    for k in (2, 8, 33):
        kn = O.knobs(g, k, 0.03, 5, 1)
        part = start_partition(g, k, k)
        bw0 = O.block_weights(g, part, k)
        ov0 = int(np.maximum(bw0.astype(np.int64) - kn.upper_bound, 0).sum())
        cut0 = O.edge_cut(g, part)
        out = O.jet_refine(g, kn, part, kn.upper_bound, level=1)
        bw = O.block_weights(g, out, k)
        ov = int(np.maximum(bw.astype(np.int64) - kn.upper_bound, 0).sum())
        cut = O.edge_cut(g, out)
        assert (ov, cut) <= (ov0, cut0)
        if ov0 == 0:
            assert ov == 0
        assert np.array_equal(out, O.jet_refine(g, kn, part, kn.upper_bound, level=1))  # deterministic


def test_jet_beats_lp_refinement(graphs):
    wins = 0
    for g, k in ((graphs.rgg2d(1 << 15, seed=0), 16), (graphs.rgg3d(1 << 14, seed=1), 8),
                 (graphs.grid2d(150, 150), 32)):
        kn = O.knobs(g, k, 0.03, 0, 0)
        kn.refinement = 0
        cut_lp, _, st_lp = O.kaffpa_knobs(g, kn)
        kn.refinement = 1
        cut_jet, part, st = O.kaffpa_knobs(g, kn)
        assert st.balanced
        wins += cut_jet < cut_lp
    assert wins == 3
