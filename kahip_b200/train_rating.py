"""Trains the learned edge rating (kahip_b200/csrc/learned.cuh) on the GPU.

Training data: seeded RGG2D / RGG3D / R-MAT graphs with n log-uniform in
[2^14, 2^16] and every level of their heavy-edge-matching hierarchy (the
graphs the rating is applied to), each labelled cut / not cut by a partition
of the plain method (this library's kaffpa, eco preset, k in {8, 64}).
Validation: held-out RGG2D n=2^17 and R-MAT n=2^15, k=64, imbalance 3%: the
cut of kaffpa with the learned-rating matching against the expansion*^2
matching.  Writes <out>.f32 (the parameters, little-endian FP32) and
<out>.json (what was trained on and how it validated).

    python -m kahip_b200.train_rating --out kahip_b200/data/rating_mpnn
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time

import numpy as np

from . import graphs, native


def label_of(g: dict, part: np.ndarray) -> np.ndarray:
    src = np.repeat(np.arange(g["n"]), np.diff(g["xadj"]))
    return (part[src] != part[g["adjncy"]]).astype(np.uint8)


def hierarchy(g: dict, k: int, seed: int, max_levels: int = 6) -> list:
    """The level graphs of g's heavy-edge-matching hierarchy (level 0 first)."""
    out = [g]
    kn = native.derive_knobs(g["n"], g["vwgt"], k, 0.03, seed, native.FAST)
    cur = g
    for level in range(max_levels):
        lab = native.hem_match(cur, kn, level)
        c, _ = native.contract(cur, lab)
        if c["n"] == 0 or cur["n"] / c["n"] < 1.1 or c["n"] < kn.num_stop:
            break
        out.append(c)
        cur = c
    return out


def base_graph(kind: int, n: int, seed: int) -> dict:
    if kind == 0:
        return graphs.rgg2d(n, seed=seed)
    if kind == 1:
        return graphs.rgg3d(n, seed=seed)
    return graphs.rmat(max(4, int(round(np.log2(n)))), samples=8 * n, seed=seed)


def build_training_set(count: int, seed: int):
    rng = np.random.default_rng(seed)
    data, desc = [], []
    for i in range(count):
        kind = i % 3
        n = int(np.exp(rng.uniform(np.log(2 ** 14), np.log(2 ** 16))))
        k = 8 if i % 2 == 0 else 64
        g = base_graph(kind, n, int(rng.integers(0, 1 << 30)))
        for lvl, h in enumerate(hierarchy(g, k, i)):
            _, _, part = native.kaffpa_ex(h["xadj"], h["adjncy"], k, 0.03, i, native.ECO, vwgt=h["vwgt"],
                                          adjwgt=h["adjwgt"])
            data.append((h, label_of(h, part)))
            desc.append({"kind": ["rgg2d", "rgg3d", "rmat"][kind], "level": lvl, "n": h["n"], "m": h["m"], "k": k})
    return data, desc


def init_params(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    P = np.zeros(native.RATING_PARAMS, np.float32)
    off = 0
    for rows, cols, bias in [(64, 2, True)] + [(64, 128, True)] * 3 + [(32, 64, True), (32, 2, False)]:
        P[off:off + rows * cols] = rng.normal(0, np.sqrt(2.0 / cols), rows * cols)
        off += rows * cols
        if bias:
            off += rows
    P[off:off + 32] = rng.normal(0, np.sqrt(1.0 / 32), 32)
    return P


def validate(P: np.ndarray) -> list:
    out = []
    for name, g in (("rgg2d_17", graphs.rgg2d(1 << 17, seed=424242)), ("rmat_15", graphs.rmat(15, seed=4242))):
        res = {"graph": name}
        for label, coarsening in (("plain", 1), ("learned", 2)):
            kn = native.derive_knobs(g["n"], g["vwgt"], 64, 0.03, 0, native.FAST)
            kn.coarsening = coarsening
            kn.rating_model = P.ctypes.data_as(ctypes.c_void_p) if coarsening == 2 else None
            _, cut, _ = native.kaffpa_knobs(g["xadj"], g["adjncy"], kn, vwgt=g["vwgt"], adjwgt=g["adjwgt"])
            res[label] = int(cut)
        res["ratio"] = res["learned"] / max(1, res["plain"])
        out.append(res)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="output path without extension")
    ap.add_argument("--graphs", type=int, default=24)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    t0 = time.time()
    data, desc = build_training_set(args.graphs, args.seed)
    t1 = time.time()
    P0 = init_params(args.seed)
    P, loss = native.rating_train(data, P0, args.steps, args.lr)
    t2 = time.time()
    val = validate(P)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    P.astype("<f4").tofile(args.out + ".f32")
    meta = {
        "params": native.RATING_PARAMS, "steps": args.steps, "lr": args.lr, "seed": args.seed,
        "training_graphs": len(data), "training_set": desc,
        "labels": "cut / not cut under this library's kaffpa (eco preset) of each level graph",
        "loss_first": float(loss[:20].mean()), "loss_last": float(loss[-20:].mean()),
        "validation": val, "validated": all(v["ratio"] <= 1.0 for v in val),
        "seconds": {"data": t1 - t0, "train": t2 - t1},
    }
    with open(args.out + ".json", "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps({k: meta[k] for k in ("training_graphs", "loss_first", "loss_last", "validation", "validated",
                                            "seconds")}))


if __name__ == "__main__":
    main()
