"""Balance repair in the oracle (CPU): from skewed starts it brings every
block to the bound, moves only vertices of overloaded blocks, and is
deterministic; the device equals the oracle (tests/test_gpu_parity.py)."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("which,k", [("rgg2d", 4), ("rgg2d", 33), ("grid", 7), ("rmat", 16), ("weighted", 9)])
def test_balance_reaches_the_bound(graphs, which, k):
    g = {"rgg2d": lambda: graphs.rgg2d(1 << 12, seed=5), "grid": lambda: graphs.grid2d(60, 50),
         "rmat": lambda: graphs.rmat(11, seed=6), "weighted": lambda: graphs.rgg2d(3000, seed=7)}[which]()
    if which == "weighted":
        g["vwgt"] = np.random.default_rng(1).integers(1, 6, g["n"]).astype(np.int32)
    kn = O.knobs(g, k, 0.03, 3, 0)
    rng = np.random.default_rng(k)
    # skewed start: half of the vertices in block 0, the rest spread
    part = rng.integers(0, k, g["n"]).astype(np.int32)
    part[rng.random(g["n"]) < 0.5] = 0
    bw0 = O.block_weights(g, part, k)
    out, ok = O.balance(g, kn, part, kn.final_bound, 0)
    bw = O.block_weights(g, out, k)
    assert ok and bw.max() <= kn.final_bound
    moved = out != part
    assert np.all(bw0[part[moved]] > kn.final_bound)  # only overloaded blocks release vertices
    assert np.array_equal(out, O.balance(g, kn, part, kn.final_bound, 0)[0])


def test_balance_leaves_a_balanced_partition_alone(graphs):
    g = graphs.rgg2d(2000, seed=2)
    kn = O.knobs(g, 8, 0.03, 0, 0)
    part = (np.arange(g["n"]) * 8 // g["n"]).astype(np.int32)
    out, ok = O.balance(g, kn, part, kn.final_bound, 0)
    assert ok and np.array_equal(out, part)
