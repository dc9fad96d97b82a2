"""Generates tests/golden/reference_outputs.npz from the reference itself.

Runs the reference KaHIP routines (oracle/_ref/libkahip_ref.so, built from
the reference sources by `make -C oracle ref`) on small seeded graphs from
kahip_b200.graphs and stores their outputs.  tests/test_golden.py checks the
CPU oracle against these vectors on machines without the reference sources.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import csr_from_edges, tie_free  # noqa: E402

from kahip_b200 import graphs  # noqa: E402
from oracle import oracle as O  # noqa: E402


def graph_set():
    rng = np.random.default_rng(0)
    out = {
        "rgg2d_2000": graphs.rgg2d(2000, seed=1),
        "rgg3d_1500": graphs.rgg3d(1500, seed=2),
        "rmat_10": graphs.rmat(10, seed=3),
        "grid_30x20": graphs.grid2d(30, 20),
    }
    g = tie_free(graphs.rgg2d(1500, seed=4))
    g["vwgt"] = rng.integers(1, 9, g["n"]).astype(np.int32)
    out["tiefree_rgg2d_1500"] = g
    return out


def fingerprint(g):
    return np.array([g["n"], g["m"], int(g["adjncy"].astype(np.int64).sum()),
                     int(g["adjwgt"].astype(np.int64).sum()), int(g["vwgt"].astype(np.int64).sum())], np.int64)


BALANCE_CASES = [(1 << 24, 64, 0.03, 0), (1 << 15, 8, 0.03, 1), (5000, 3, 0.0, 0), (777, 256, 0.05, 2),
                 (100, 7, 0.1, 3), (1 << 20, 2, 0.001, 4), (12345, 17, 0.2, 5)]


def main():
    assert O.ref_available(), "build the reference first: make -C oracle ref"
    d = {}
    d["balance_cases"] = np.array(BALANCE_CASES, dtype=np.float64)
    d["balance_out"] = np.array([O.ref_balance_config(n, None, k, imb, mode) for n, k, imb, mode in BALANCE_CASES],
                                np.int64)
    for name, g in graph_set().items():
        d[f"{name}/fingerprint"] = fingerprint(g)
        d[f"{name}/rating"] = O.ref_rating(g)
        rng = np.random.default_rng(1)
        parts = np.stack([rng.integers(0, k, g["n"]).astype(np.int32) for k in (2, 5, 64)])
        d[f"{name}/cut_parts"] = parts
        d[f"{name}/cut"] = np.array([O.ref_edge_cut(g, p, k) for p, k in zip(parts, (2, 5, 64))], np.int64)
        d[f"{name}/balance"] = np.array([O.ref_balance(g, p, k) for p, k in zip(parts, (2, 5, 64))])
        lab = rng.integers(0, g["n"] // 7 + 1, g["n"]).astype(np.int32)
        c, cmap = O.ref_contract_clustering(g, lab)
        c = O.canonical(c)
        d[f"{name}/contract_label"] = lab
        d[f"{name}/contract_cmap"] = cmap
        for key in ("xadj", "adjncy", "adjwgt", "vwgt"):
            d[f"{name}/contract_{key}"] = c[key]
        if name.startswith("tiefree"):
            order = O.ref_degree_order(g)
            d[f"{name}/order"] = order
            for bound, rounds in [(40, 1), (200, 10)]:
                d[f"{name}/lpc_{bound}_{rounds}"] = O.ref_lp_cluster(g, bound, rounds)
            k = 8
            cuts = np.sort(np.random.default_rng(k).integers(0, g["n"], k - 1))
            part = np.searchsorted(cuts, np.arange(g["n"]), side="right").astype(np.int32)
            d[f"{name}/lpr_part0"] = part
            W = int(g["vwgt"].sum())
            bound = int(1.03 * np.ceil(W / k))
            d[f"{name}/lpr_bound"] = np.array([bound])
            d[f"{name}/lpr_out"] = O.ref_lp_refine(g, k, bound, 25, part)
        if name == "rgg2d_2000":
            d[f"{name}/kaffpa_cut_fast_k8"] = np.array([O.ref_kaffpa(g, 8, 0.03, 0, 0)[0]])
            d[f"{name}/kaffpa_cut_eco_k8"] = np.array([O.ref_kaffpa(g, 8, 0.03, 0, 1)[0]])
    big = graphs.rgg2d(1 << 18, seed=0)
    d["rgg2d_18/fingerprint"] = fingerprint(big)
    for k in (8, 64):
        d[f"rgg2d_18/kaffpa_cut_fast_k{k}"] = np.array([O.ref_kaffpa(big, k, 0.03, 0, 0)[0]])
    five = csr_from_edges(5, [(0, 1), (0, 4), (1, 2), (1, 4), (2, 3), (3, 4)])
    d["interface_test/eco_k2_cut"] = np.array([O.ref_kaffpa(five, 2, 0.03, 0, 1)[0]])
    out = os.path.join(HERE, "reference_outputs.npz")
    np.savez_compressed(out, **d)
    print(f"wrote {out} ({os.path.getsize(out)} bytes, {len(d)} arrays)")


if __name__ == "__main__":
    main()
