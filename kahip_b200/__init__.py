"""B200-native KaFFPa: drop-in replacement for the kaffpa() path of KaHIP.

Python interface mirroring the reference's ``kahip`` module
(misc/pymodule/kahip.cpp:4-47, python/kahip/__init__.py):

    edgecut, blocks = kahip_b200.kaffpa(vwgt, xadj, adjcwgt, adjncy, nparts,
                                        imbalance, suppress_output, seed, mode)

Same argument meaning (imbalance is a fraction, mode FAST=0 / ECO=1 / ...),
same return value (edge cut, list of block ids).  The call goes through the
C ABI of libkahip_b200.so to the GPU; it raises KaHIPError where the
reference would have undefined behaviour (invalid CSR) and when no CUDA
device is present.
"""
from __future__ import annotations

from . import native
from .native import (ECO, ECOSOCIAL, FAST, FASTSOCIAL, STRONG, STRONGSOCIAL, KaHIPError, Knobs, Stats,
                     derive_knobs, kaffpa_ex)

__all__ = ["kaffpa", "kaffpa_ex", "kahip_graph", "KaHIPError", "Knobs", "Stats", "derive_knobs", "native",
           "FAST", "ECO", "STRONG", "FASTSOCIAL", "ECOSOCIAL", "STRONGSOCIAL"]


def kaffpa(vwgt, xadj, adjcwgt, adjncy, nparts, imbalance, suppress_output=True, seed=0, mode=FAST):
    """Partition a graph into nparts blocks; returns (edgecut, blocks)."""
    _, cut, part = kaffpa_ex(xadj, adjncy, nparts, imbalance, seed, mode,
                             vwgt=None if vwgt is None or len(vwgt) == 0 else vwgt,
                             adjwgt=None if adjcwgt is None or len(adjcwgt) == 0 else adjcwgt)
    return int(cut), part.tolist()


class kahip_graph:
    """Builds a CSR graph from undirected edges (as python/kahip/__init__.py's
    helper of the same name does)."""

    def __init__(self):
        self.num_nodes = 0
        self.edges = {}
        self.node_weights = {}

    def set_num_nodes(self, n):
        self.num_nodes = n
        for i in range(n):
            self.node_weights.setdefault(i, 1)

    def add_undirected_edge(self, source, target, weight=1):
        if source >= self.num_nodes or target >= self.num_nodes:
            raise ValueError(f"Node index out of range. Graph has {self.num_nodes} nodes.")
        if source == target:
            return
        self.edges[(source, target)] = weight
        self.edges[(target, source)] = weight

    def set_weight(self, node, weight):
        self.node_weights[node] = weight

    def get_csr_arrays(self):
        rows = [[] for _ in range(self.num_nodes)]
        for (s, t), w in self.edges.items():
            rows[s].append((t, w))
        xadj, adjncy, adjcwgt = [0], [], []
        for r in rows:
            r.sort()
            adjncy += [t for t, _ in r]
            adjcwgt += [w for _, w in r]
            xadj.append(len(adjncy))
        vwgt = [self.node_weights.get(i, 1) for i in range(self.num_nodes)]
        return vwgt, xadj, adjcwgt, adjncy
