import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity of the CUDA path vs the oracle")
    config.addinivalue_line("markers", "slow: larger sizes")


@pytest.fixture(scope="session")
def graphs():
    from kahip_b200 import graphs as G
    return G


def csr_from_edges(n, edges, weights=None, vwgt=None):
    """Symmetric CSR (rows sorted) from undirected edges [(u, v), ...]."""
    rows = [dict() for _ in range(n)]
    for i, (u, v) in enumerate(edges):
        if u == v:
            continue
        w = 1 if weights is None else weights[i]
        rows[u][v] = rows[u].get(v, 0) + w
        rows[v][u] = rows[v].get(u, 0) + w
    xadj = [0]
    adj, wgt = [], []
    for r in rows:
        for t in sorted(r):
            adj.append(t)
            wgt.append(r[t])
        xadj.append(len(adj))
    from kahip_b200.graphs import from_csr
    return from_csr(np.array(xadj), np.array(adj, dtype=np.int32), np.array(wgt, dtype=np.int32),
                    None if vwgt is None else np.array(vwgt, dtype=np.int32))


def tie_free(g, seed=7):
    """Same structure, random 20-bit edge weights (symmetric), so that label
    propagation never meets two equally connected candidates."""
    rng = np.random.default_rng(seed)
    n, xadj, adj = g["n"], g["xadj"], g["adjncy"]
    src = np.repeat(np.arange(n), np.diff(xadj))
    lo = np.minimum(src, adj).astype(np.int64)
    hi = np.maximum(src, adj).astype(np.int64)
    key = lo * n + hi
    uniq, inv = np.unique(key, return_inverse=True)
    w = rng.integers(1 << 10, 1 << 20, size=len(uniq)).astype(np.int32)
    out = dict(g)
    out["adjwgt"] = w[inv]
    return out
