"""Generates tests/golden/scale_digests.json: the CPU oracle's results at the
sizes the benchmark configurations name, so that the GPU parity test
(tests/test_gpu_scale.py) can check the device path bit for bit at those
sizes without rerunning the oracle (minutes of single-threaded CPU work per
graph) on every test run.

Per configuration it records the input graph's sha256 (so a generator change
is caught before any partition is compared), the edge cut, the sha256 of
part[] (int32, little endian), the initial partition's cut and per level the
node count, directed entry count, cut and heaviest block.

    python tests/golden/make_scale_digests.py [--jobs J] [--only NAME ...]

The oracle (oracle/liboracle.so, built by `make -C oracle`) is test
infrastructure; this script runs only on the CPU.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden", "scale_digests.json")

FAST, ECO = 0, 1

# (graph kind, log2 n) -> [(k, seed, mode), ...]
CONFIGS = {
    # the reference's own CPU-runnable size (RGG2D n=2^15), its headline tuple first
    ("rgg2d", 15): [(8, 0, FAST), (64, 0, FAST), (8, 0, ECO), (64, 0, ECO)],
    # the single-GPU headline graph: k in {16, 64, 256}, seeds 0-4, plus eco at k=64
    ("rgg2d", 24): [(k, s, FAST) for k in (16, 64, 256) for s in range(5)] + [(64, 0, ECO)],
    ("rgg3d", 22): [(k, 0, FAST) for k in (16, 64, 256)],
    ("rmat", 23): [(64, 0, FAST), (256, 0, FAST)],
}


def make_graph(kind: str, logn: int) -> dict:
    from kahip_b200 import graphs
    if kind == "rgg2d":
        return graphs.rgg2d(1 << logn, seed=0)
    if kind == "rgg3d":
        return graphs.rgg3d(1 << logn, seed=0)
    return graphs.rmat(logn, seed=0)


def unit_weights(kind: str) -> bool:
    # the geometric graphs are passed with NULL weights (unit), R-MAT with its
    # duplicate-multiplicity edge weights
    return kind != "rmat"


def graph_sha256(g: dict) -> str:
    h = hashlib.sha256()
    for key in ("xadj", "adjncy", "adjwgt", "vwgt"):
        h.update(g[key].astype("<i4", copy=False).tobytes())
    return h.hexdigest()


def config_name(kind: str, logn: int, k: int, seed: int, mode: int) -> str:
    return f"{kind}_2p{logn}_k{k}_s{seed}_{'fast' if mode == FAST else 'eco'}"


def _run(task):
    kind, logn, runs = task
    sys.path.insert(0, ROOT)
    import numpy as np

    from oracle import oracle
    g = make_graph(kind, logn)
    gsha = graph_sha256(g)
    out = {}
    for k, seed, mode in runs:
        t = time.perf_counter()
        cut, part, st = oracle.kaffpa(g, k, 0.03, seed, mode, unit_weights=unit_weights(kind))
        secs = time.perf_counter() - t
        kn = oracle.knobs(g, k, 0.03, seed, mode)
        bw = oracle.block_weights(g, part, k)
        out[config_name(kind, logn, k, seed, mode)] = {
            "graph": kind, "logn": logn, "n": g["n"], "m_directed": g["m"], "graph_sha256": gsha,
            "k": k, "seed": seed, "mode": mode, "imbalance": 0.03,
            "cut": int(cut), "part_sha256": hashlib.sha256(part.astype("<i4").tobytes()).hexdigest(),
            "max_block": int(bw.max()), "bound": int(kn.final_bound),
            "initial_cut": int(st.initial_cut),
            "levels": [[int(st.level_n[i]), int(st.level_m[i]), int(st.level_cut[i]), int(st.level_maxbw[i])]
                       for i in range(st.levels)],
            "oracle_seconds": round(secs, 1),
        }
        print(f"{config_name(kind, logn, k, seed, mode)}: cut {cut} ({secs:.1f} s)", flush=True)
        del part
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=4)
    ap.add_argument("--only", nargs="*", help="graph keys such as rgg2d_2p24")
    a = ap.parse_args()
    tasks = []
    for (kind, logn), runs in CONFIGS.items():
        if a.only and f"{kind}_2p{logn}" not in a.only:
            continue
        # split the long lists so that several processes share one graph size
        step = 4 if logn >= 22 else len(runs)
        for i in range(0, len(runs), step):
            tasks.append((kind, logn, runs[i:i + step]))
    tasks.sort(key=lambda t: -t[1] * len(t[2]))
    results = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            results = json.load(f)["configs"]
    with mp.get_context("spawn").Pool(a.jobs) as pool:
        for out in pool.imap_unordered(_run, tasks):
            results.update(out)
            with open(OUT, "w") as f:
                json.dump({"generator": "tests/golden/make_scale_digests.py",
                           "oracle": "oracle/liboracle.so (C restatement of the deterministic schedule)",
                           "configs": dict(sorted(results.items()))}, f, indent=1)


if __name__ == "__main__":
    main()
