"""ctypes bindings of the checkers -- TEST INFRASTRUCTURE ONLY.

* liboracle.so      : the C restatement of the deterministic schedule.
* _ref/libkahip_ref.so : the reference KaHIP library compiled from its own
  sources by oracle/Makefile (present only where the reference sources were
  available at build time), with ref_harness.cpp's single-routine entry points.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_OR = None
_REF = None

c_int_p = ctypes.POINTER(ctypes.c_int)


class Knobs(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int), ("imbalance", ctypes.c_double), ("seed", ctypes.c_int),
                ("mode", ctypes.c_int), ("total_weight", ctypes.c_uint32),
                ("upper_bound", ctypes.c_uint32), ("final_bound", ctypes.c_uint32),
                ("num_stop", ctypes.c_uint32), ("max_vertex_weight", ctypes.c_uint32),
                ("cluster_bound", ctypes.c_uint32),
                ("lpc_rounds", ctypes.c_int), ("lpc_subrounds", ctypes.c_int),
                ("ref_rounds", ctypes.c_int), ("ref_subrounds", ctypes.c_int),
                ("ref_classes", ctypes.c_int), ("bal_iters", ctypes.c_int),
                ("ip_reps", ctypes.c_int), ("ip_tries", ctypes.c_int),
                ("ip_fm_passes", ctypes.c_int), ("ip_fm_stall", ctypes.c_int),
                ("max_levels", ctypes.c_int), ("coarsening", ctypes.c_int),
                ("match_rounds", ctypes.c_int), ("rating_model", ctypes.c_void_p),
                ("rating_fallback", ctypes.c_double), ("rating_levels", ctypes.c_int),
                ("refinement", ctypes.c_int), ("jet_iters", ctypes.c_int), ("jet_patience", ctypes.c_int),
                ("jet_c0", ctypes.c_int), ("jet_c", ctypes.c_int), ("ip_mode", ctypes.c_int),
                ("ip_jet_iters", ctypes.c_int), ("ip_jet_patience", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int), ("level_n", ctypes.c_int * 64),
                ("level_m", ctypes.c_longlong * 64), ("level_cut", ctypes.c_longlong * 64),
                ("level_maxbw", ctypes.c_uint32 * 64), ("initial_cut", ctypes.c_longlong),
                ("balanced", ctypes.c_int)]


class Graph(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("xadj", c_int_p), ("adjncy", c_int_p),
                ("adjwgt", c_int_p), ("vwgt", c_int_p)]


def _p(a):
    return a.ctypes.data_as(c_int_p) if a is not None else None


def lib():
    global _OR
    if _OR is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        L.or_edge_cut.restype = ctypes.c_longlong
        L.or_balance_ratio.restype = ctypes.c_double
        L.or_lp_cluster_seq.restype = ctypes.c_int
        L.or_contract.restype = ctypes.c_int
        L.or_balance.restype = ctypes.c_int
        L.or_kaffpa.restype = ctypes.c_int
        L.or_kaffpa_knobs.restype = ctypes.c_int
        L.or_kaffpa_combine.restype = ctypes.c_int
        L.or_kaffpae.restype = ctypes.c_int
        L.or_hash.restype = ctypes.c_uint32
        L.or_hash.argtypes = [ctypes.c_uint64, ctypes.c_uint32]
        L.or_stream.restype = ctypes.c_uint64
        L.or_stream.argtypes = [ctypes.c_int] * 4
        L.or_mix64.restype = ctypes.c_uint64
        L.or_mix64.argtypes = [ctypes.c_uint64]
        _OR = L
    return _OR


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libkahip_ref.so"))


def ref():
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libkahip_ref.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/_ref/libkahip_ref.so missing: run `make -C oracle ref`")
        L = ctypes.CDLL(path)
        L.ref_edge_cut.restype = ctypes.c_int
        L.ref_balance.restype = ctypes.c_double
        L.ref_stop_rule_continue.restype = ctypes.c_int
        _REF = L
    return _REF


class G:
    """Keeps numpy arrays alive behind an or_graph struct."""

    def __init__(self, g: dict):
        self.d = {k: (np.ascontiguousarray(v, np.int32) if isinstance(v, np.ndarray) else v)
                  for k, v in g.items()}
        d = self.d
        self.s = Graph(d["n"], _p(d["xadj"]), _p(d["adjncy"]), _p(d["adjwgt"]), _p(d["vwgt"]))

    @property
    def ref(self):
        return ctypes.byref(self.s)


# ------------------------------------------------------------------ oracle

def knobs(g: dict, k: int, imbalance=0.03, seed=0, mode=0) -> Knobs:
    kn = Knobs()
    lib().or_derive_knobs(g["n"], _p(g["vwgt"]), k, ctypes.c_double(imbalance), seed, mode,
                          ctypes.byref(kn))
    return kn


def stop_continue(kn: Knobs, nf: int, nc: int) -> bool:
    return bool(lib().or_stop_continue(ctypes.byref(kn), nf, nc))


def balance_ratio(g: dict, part, k: int) -> float:
    return lib().or_balance_ratio(G(g).ref, _p(np.ascontiguousarray(part, np.int32)), k)


def edge_cut(g: dict, part) -> int:
    return lib().or_edge_cut(G(g).ref, _p(np.ascontiguousarray(part, np.int32)))


def stream(seed: int, tag: int, level: int, rnd: int) -> int:
    return int(lib().or_stream(seed, tag, level, rnd))


def hash32(ks: int, x: int) -> int:
    return int(lib().or_hash(ctypes.c_uint64(ks), ctypes.c_uint32(x & 0xFFFFFFFF)))


def block_weights(g: dict, part, k: int) -> np.ndarray:
    bw = np.zeros(k, np.uint32)
    lib().or_block_weights(G(g).ref, _p(np.ascontiguousarray(part, np.int32)), k,
                           bw.ctypes.data_as(ctypes.c_void_p))
    return bw


def rating(g: dict) -> np.ndarray:
    out = np.empty(g["m"], np.float64)
    lib().or_rate_expansion_star_2(G(g).ref, out.ctypes.data_as(ctypes.c_void_p))
    return out


def lp_cluster(g: dict, kn: Knobs, level=0) -> np.ndarray:
    lab = np.empty(g["n"], np.int32)
    lib().or_lp_cluster(G(g).ref, ctypes.byref(kn), level, _p(lab))
    return lab


def hem_match(g: dict, kn: Knobs, level=0, rating_q=None) -> np.ndarray:
    """Heavy-edge matching labels of one level (min(v, mate) or v)."""
    lab = np.empty(g["n"], np.int32)
    rq = None if rating_q is None else np.ascontiguousarray(rating_q, np.uint32)
    lib().or_hem_match(G(g).ref, ctypes.byref(kn), level,
                       None if rq is None else rq.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), _p(lab))
    return lab


def lp_cluster_seq(g: dict, bound: int, rounds: int, order) -> np.ndarray:
    lab = np.empty(g["n"], np.int32)
    lib().or_lp_cluster_seq(G(g).ref, ctypes.c_uint32(bound), rounds,
                            _p(np.ascontiguousarray(order, np.int32)), _p(lab))
    return lab


def contract(g: dict, label) -> tuple[dict, np.ndarray]:
    n, m = g["n"], g["m"]
    cmap = np.empty(n, np.int32)
    cx = np.empty(n + 1, np.int32)
    ca = np.empty(max(m, 1), np.int32)
    cw = np.empty(max(m, 1), np.int32)
    cv = np.empty(max(n, 1), np.int32)
    nc = lib().or_contract(G(g).ref, _p(np.ascontiguousarray(label, np.int32)), _p(cmap), _p(cx),
                           _p(ca), _p(cw), _p(cv))
    mc = int(cx[nc])
    return dict(n=nc, m=mc, xadj=cx[:nc + 1].copy(), adjncy=ca[:mc].copy(), adjwgt=cw[:mc].copy(),
                vwgt=cv[:nc].copy()), cmap


def jet_refine(g: dict, kn: Knobs, part, bound: int, level=0) -> np.ndarray:
    p = np.array(part, np.int32)
    lib().or_jet_refine(G(g).ref, ctypes.byref(kn), level, ctypes.c_uint32(bound), _p(p))
    return p


def lp_refine(g: dict, kn: Knobs, part, bound: int, level=0) -> np.ndarray:
    p = np.array(part, np.int32)
    lib().or_lp_refine(G(g).ref, ctypes.byref(kn), level, ctypes.c_uint32(bound), _p(p))
    return p


def lp_refine_seq(g: dict, k: int, bound: int, rounds: int, order, part) -> np.ndarray:
    p = np.array(part, np.int32)
    lib().or_lp_refine_seq(G(g).ref, k, ctypes.c_uint32(bound), rounds,
                           _p(np.ascontiguousarray(order, np.int32)), _p(p))
    return p


def balance(g: dict, kn: Knobs, part, bound: int, level=0) -> tuple[np.ndarray, int]:
    p = np.array(part, np.int32)
    ok = lib().or_balance(G(g).ref, ctypes.byref(kn), level, ctypes.c_uint32(bound), _p(p))
    return p, ok


def initial_partition(g: dict, kn: Knobs) -> np.ndarray:
    p = np.empty(g["n"], np.int32)
    lib().or_initial_partition(G(g).ref, ctypes.byref(kn), _p(p))
    return p


def initial_partition_batched(g: dict, kn: Knobs) -> np.ndarray:
    """The batched recursive bisection (the device's initial partitioner)."""
    p = np.empty(g["n"], np.int32)
    lib().or_initial_partition_batched(G(g).ref, ctypes.byref(kn), _p(p))
    return p


def kaffpa(g: dict, k: int, imbalance=0.03, seed=0, mode=0, unit_weights=False):
    """Returns (edgecut, part, stats)."""
    part = np.empty(g["n"], np.int32)
    cut = ctypes.c_longlong()
    st = Stats()
    rc = lib().or_kaffpa(g["n"], None if unit_weights else _p(g["vwgt"]), _p(g["xadj"]),
                         None if unit_weights else _p(g["adjwgt"]), _p(g["adjncy"]), k,
                         ctypes.c_double(imbalance), seed, mode, ctypes.byref(cut), _p(part),
                         ctypes.byref(st))
    if rc != 0:
        raise ValueError(f"or_kaffpa rejected the input ({rc})")
    return cut.value, part, st


def kaffpa_knobs(g: dict, kn: Knobs, unit_weights=False):
    """Whole schedule with explicit knobs.  Returns (edgecut, part, stats)."""
    part = np.empty(g["n"], np.int32)
    cut = ctypes.c_longlong()
    st = Stats()
    rc = lib().or_kaffpa_knobs(g["n"], None if unit_weights else _p(g["vwgt"]), _p(g["xadj"]),
                               None if unit_weights else _p(g["adjwgt"]), _p(g["adjncy"]), ctypes.byref(kn),
                               ctypes.byref(cut), _p(part), ctypes.byref(st))
    if rc != 0:
        raise ValueError(f"or_kaffpa_knobs rejected the input ({rc})")
    return cut.value, part, st


def kaffpae(g: dict, kn: Knobs, population: int, generations: int, per_generation: int, unit_weights=False):
    """KaFFPaE-style evolution (oracle.c or_kaffpae).  Returns (edgecut, part, history)."""
    part = np.empty(g["n"], np.int32)
    hist = np.zeros(generations + 1, np.int64)
    cut = ctypes.c_longlong()
    rc = lib().or_kaffpae(g["n"], None if unit_weights else _p(g["vwgt"]), _p(g["xadj"]),
                          None if unit_weights else _p(g["adjwgt"]), _p(g["adjncy"]), ctypes.byref(kn),
                          population, generations, per_generation, ctypes.byref(cut), _p(part),
                          hist.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
    if rc != 0:
        raise ValueError(f"or_kaffpae rejected the input ({rc})")
    return cut.value, part, hist


def kaffpa_combine(g: dict, kn: Knobs, part_a, part_b, unit_weights=False):
    """KaFFPaE combine of two partitions (oracle.c or_kaffpa_combine).
    Returns (edgecut, part, stats)."""
    part = np.empty(g["n"], np.int32)
    pa = np.ascontiguousarray(part_a, dtype=np.int32)
    pb = np.ascontiguousarray(part_b, dtype=np.int32)
    cut = ctypes.c_longlong()
    st = Stats()
    rc = lib().or_kaffpa_combine(g["n"], None if unit_weights else _p(g["vwgt"]), _p(g["xadj"]),
                                 None if unit_weights else _p(g["adjwgt"]), _p(g["adjncy"]), ctypes.byref(kn),
                                 _p(pa), _p(pb), ctypes.byref(cut), _p(part), ctypes.byref(st))
    if rc != 0:
        raise ValueError(f"or_kaffpa_combine rejected the input ({rc})")
    return cut.value, part, st


# --------------------------------------------------------------- reference

def ref_read_metis(path: str) -> dict:
    """graph_io::readGraphWeighted of the reference, as a CSR dict (run in a
    separate process: oracle/_ref/ref_read_metis)."""
    import subprocess
    import tempfile
    exe = os.path.join(HERE, "_ref", "ref_read_metis")
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "csr.bin")
        subprocess.run([exe, path, out], check=True)
        raw = open(out, "rb").read()
    n = int(np.frombuffer(raw[:4], np.int32)[0])
    m = int(np.frombuffer(raw[4:12], np.int64)[0])
    a = np.frombuffer(raw[12:], np.int32)
    x, a = a[:n + 1], a[n + 1:]
    adj, a = a[:m], a[m:]
    w, v = a[:m], a[m:m + n]
    return dict(n=n, m=m, xadj=x.copy(), adjncy=adj.copy(), adjwgt=w.copy(), vwgt=v.copy())


def ref_kaffpa(g: dict, k: int, imbalance=0.03, seed=0, mode=0):
    """Reference kaffpa() from the library built out of the reference sources."""
    L = ref()
    n = ctypes.c_int(g["n"])
    kk = ctypes.c_int(k)
    imb = ctypes.c_double(imbalance)
    cut = ctypes.c_int()
    part = np.empty(g["n"], np.int32)
    L.kaffpa(ctypes.byref(n), _p(g["vwgt"]), _p(g["xadj"]), _p(g["adjwgt"]), _p(g["adjncy"]),
             ctypes.byref(kk), ctypes.byref(imb), ctypes.c_bool(True), seed, mode,
             ctypes.byref(cut), _p(part))
    return cut.value, part


def ref_balance_config(n: int, vwgt, k: int, imbalance=0.03, mode=0):
    u, ns, mv = ctypes.c_uint(), ctypes.c_uint(), ctypes.c_uint()
    ref().ref_balance_config(n, _p(vwgt), k, ctypes.c_double(imbalance), mode, ctypes.byref(u),
                             ctypes.byref(ns), ctypes.byref(mv))
    return u.value, ns.value, mv.value


def ref_stop_continue(nf: int, nc: int, n0: int, k: int, work_load: int) -> bool:
    return bool(ref().ref_stop_rule_continue(ctypes.c_uint(nf), ctypes.c_uint(nc), n0, k,
                                             ctypes.c_uint(work_load)))


def ref_edge_cut(g: dict, part, k: int) -> int:
    return ref().ref_edge_cut(g["n"], _p(g["xadj"]), _p(g["adjncy"]), _p(g["adjwgt"]),
                              _p(np.ascontiguousarray(part, np.int32)), k)


def ref_balance(g: dict, part, k: int) -> float:
    return ref().ref_balance(g["n"], _p(g["xadj"]), _p(g["adjncy"]), _p(g["vwgt"]),
                             _p(np.ascontiguousarray(part, np.int32)), k)


def ref_rating(g: dict) -> np.ndarray:
    out = np.empty(g["m"], np.float64)
    ref().ref_rate_expansion_star_2(g["n"], _p(g["xadj"]), _p(g["adjncy"]), _p(g["vwgt"]),
                                    _p(g["adjwgt"]), out.ctypes.data_as(ctypes.c_void_p))
    return out


def _ref_contract(fn, g, arr):
    n, m = g["n"], g["m"]
    nc = ctypes.c_int()
    cx = np.empty(n + 1, np.int32)
    ca = np.empty(max(m, 1), np.int32)
    cw = np.empty(max(m, 1), np.int32)
    cv = np.empty(max(n, 1), np.int32)
    cmap = np.empty(n, np.int32)
    fn(n, _p(g["xadj"]), _p(g["adjncy"]), _p(g["vwgt"]), _p(g["adjwgt"]),
       _p(np.ascontiguousarray(arr, np.int32)), ctypes.byref(nc), _p(cx), _p(ca), _p(cw), _p(cv),
       _p(cmap))
    k = nc.value
    mc = int(cx[k])
    return dict(n=k, m=mc, xadj=cx[:k + 1].copy(), adjncy=ca[:mc].copy(), adjwgt=cw[:mc].copy(),
                vwgt=cv[:k].copy()), cmap


def ref_contract_clustering(g: dict, cluster):
    return _ref_contract(ref().ref_contract_clustering, g, cluster)


def ref_contract_matching(g: dict, match):
    return _ref_contract(ref().ref_contract_matching, g, match)


def ref_degree_order(g: dict) -> np.ndarray:
    o = np.empty(g["n"], np.int32)
    ref().ref_degree_order(g["n"], _p(g["xadj"]), _p(g["adjncy"]), _p(o))
    return o


def ref_lp_cluster(g: dict, bound: int, iterations: int) -> np.ndarray:
    out = np.empty(g["n"], np.int32)
    nb = ctypes.c_int()
    ref().ref_lp_cluster(g["n"], _p(g["xadj"]), _p(g["adjncy"]), _p(g["vwgt"]), _p(g["adjwgt"]),
                         ctypes.c_uint(bound), iterations, _p(out), ctypes.byref(nb))
    return out


def ref_lp_refine(g: dict, k: int, bound: int, iterations: int, part) -> np.ndarray:
    p = np.array(part, np.int32)
    ref().ref_lp_refine(g["n"], _p(g["xadj"]), _p(g["adjncy"]), _p(g["vwgt"]), _p(g["adjwgt"]), k,
                        ctypes.c_uint(bound), iterations, _p(p))
    return p


def canonical(g: dict) -> dict:
    """Rows sorted by target (for comparing graphs whose row order differs)."""
    xadj, adj, w = g["xadj"], g["adjncy"].copy(), g["adjwgt"].copy()
    for v in range(g["n"]):
        s, e = xadj[v], xadj[v + 1]
        o = np.argsort(adj[s:e], kind="stable")
        adj[s:e] = adj[s:e][o]
        w[s:e] = w[s:e][o]
    return dict(g, adjncy=adj, adjwgt=w)
