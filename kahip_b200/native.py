"""ctypes bindings of libkahip_b200.so (the C ABI in include/kahip_b200.h and
include/kaHIP_interface.h).

The library is loaded from the package directory (built in-tree by
``kahip_b200/csrc/Makefile``).  Loading needs no GPU; every compute entry
point fails with KB200_ERR_NO_DEVICE when no CUDA device is visible -- there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkahip_b200.so")

OK, ERR_INVALID_INPUT, ERR_CUDA, ERR_NO_DEVICE, ERR_OUT_OF_MEMORY, ERR_INTERNAL = 0, -1, -2, -3, -4, -5
WARN_IMBALANCED = 1

FAST, ECO, STRONG, FASTSOCIAL, ECOSOCIAL, STRONGSOCIAL = range(6)

c_int_p = ctypes.POINTER(ctypes.c_int)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)
c_ll_p = ctypes.POINTER(ctypes.c_longlong)


class Knobs(ctypes.Structure):
    """kb200_knobs"""
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

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Stats(ctypes.Structure):
    """kb200_stats"""
    _fields_ = [("levels", ctypes.c_int), ("level_n", ctypes.c_int * 64),
                ("level_m", ctypes.c_longlong * 64), ("level_cut", ctypes.c_longlong * 64),
                ("level_maxbw", ctypes.c_uint32 * 64), ("initial_cut", ctypes.c_longlong),
                ("balanced", ctypes.c_int), ("collect_level_cuts", ctypes.c_int),
                ("timing", ctypes.c_int), ("ms_total", ctypes.c_double), ("ms_h2d", ctypes.c_double),
                ("ms_coarsen", ctypes.c_double), ("ms_initial", ctypes.c_double),
                ("ms_uncoarsen", ctypes.c_double), ("ms_d2h", ctypes.c_double),
                ("nfamilies", ctypes.c_int), ("family_name", (ctypes.c_char * 24) * 32),
                ("family_ms", ctypes.c_double * 32), ("family_bytes", ctypes.c_double * 32),
                ("family_launches", ctypes.c_longlong * 32), ("sweep_vertices", ctypes.c_longlong),
                ("sweep_edges", ctypes.c_longlong), ("sweep_overflow_vertices", ctypes.c_longlong),
                ("device_bytes_peak", ctypes.c_size_t), ("rating_fallback_used", ctypes.c_int)]

    def families(self) -> dict:
        return {self.family_name[i].value.decode(): dict(ms=self.family_ms[i], bytes=self.family_bytes[i],
                                                         launches=self.family_launches[i])
                for i in range(self.nfamilies)}

    def levels_list(self):
        return [dict(n=self.level_n[i], m=self.level_m[i], cut=self.level_cut[i],
                     maxbw=self.level_maxbw[i]) for i in range(self.levels)]


RATING_PARAMS = 27137


class TrainGraph(ctypes.Structure):
    """kb200_train_graph"""
    _fields_ = [("n", ctypes.c_int), ("xadj", ctypes.c_void_p), ("adjncy", ctypes.c_void_p),
                ("adjwgt", ctypes.c_void_p), ("vwgt", ctypes.c_void_p), ("label", ctypes.c_void_p)]


class BatchItem(ctypes.Structure):
    """kb200_batch_item"""
    _fields_ = [("n", ctypes.c_int), ("xadj", ctypes.c_void_p), ("adjncy", ctypes.c_void_p),
                ("adjwgt", ctypes.c_void_p), ("vwgt", ctypes.c_void_p), ("nparts", ctypes.c_int),
                ("imbalance", ctypes.c_double), ("seed", ctypes.c_int), ("mode", ctypes.c_int),
                ("part", ctypes.c_void_p), ("edgecut", ctypes.c_longlong), ("status", ctypes.c_int)]


class BatchReport(ctypes.Structure):
    """kb200_batch_report"""
    _fields_ = [("workers", ctypes.c_int), ("failed", ctypes.c_int), ("ms_total", ctypes.c_double)]


EXPORTS = [
    # extended ABI (include/kahip_b200.h)
    "kb200_derive_knobs", "kb200_kaffpa", "kb200_kaffpa_device", "kb200_kaffpa_knobs", "kb200_kaffpa_combine",
    "kb200_kaffpae",
    "kb200_kaffpa_device_knobs", "kb200_kaffpa_batch", "kb200_kaffpa_population", "kb200_hem_match",
    "kb200_rating_infer", "kb200_rating_train", "kb200_rating_grad",
    "kb200_read_metis", "kb200_read_bgf", "kb200_write_partition", "kb200_free", "kb200_io_error",
    "kb200_lp_cluster", "kb200_contract", "kb200_jet_refine",
    "kb200_lp_refine", "kb200_balance", "kb200_edge_cut", "kb200_project", "kb200_initial_partition",
    "kb200_initial_partition_device",
    "kb200_last_error", "kb200_kernel_launches", "kb200_device_count", "kb200_edge_cut_noalloc",
    # reference-compatible ABI (include/kaHIP_interface.h)
    "kaffpa", "kaffpa_balance", "kaffpa_balance_NE", "process_mapping", "node_separator", "reduced_nd",
    "edge_partitioning",
]

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C kahip_b200/csrc`")
        L = ctypes.CDLL(LIB_PATH)
        i, vp, d, u32 = ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_uint32
        L.kb200_derive_knobs.argtypes = [i, vp, i, d, i, i, ctypes.POINTER(Knobs)]
        L.kb200_kaffpa.argtypes = [i, vp, vp, vp, vp, i, d, i, i, c_ll_p, vp, ctypes.POINTER(Stats)]
        L.kb200_kaffpa_device.argtypes = [i, vp, vp, vp, vp, i, d, i, i, c_ll_p, vp, vp, ctypes.POINTER(Stats)]
        L.kb200_kaffpa_knobs.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), c_ll_p, vp,
                                         ctypes.POINTER(Stats)]
        L.kb200_kaffpa_device_knobs.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), c_ll_p, vp, vp,
                                                ctypes.POINTER(Stats)]
        L.kb200_kaffpa_combine.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), vp, vp, c_ll_p, vp,
                                           ctypes.POINTER(Stats)]
        L.kb200_kaffpae.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), i, i, i, i, c_ll_p, vp, vp]
        L.kb200_hem_match.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), i, vp, vp]
        L.kb200_rating_infer.argtypes = [i, vp, vp, vp, vp, vp, i, vp, vp]
        L.kb200_rating_train.argtypes = [ctypes.POINTER(TrainGraph), i, i, ctypes.c_float, vp, vp]
        L.kb200_rating_grad.argtypes = [ctypes.POINTER(TrainGraph), vp, vp, vp]
        pp = ctypes.POINTER(ctypes.c_void_p)
        L.kb200_read_metis.argtypes = [ctypes.c_char_p, c_int_p, c_ll_p, pp, pp, pp, pp]
        L.kb200_read_bgf.argtypes = [ctypes.c_char_p, c_int_p, c_ll_p, pp, pp, pp, pp]
        L.kb200_write_partition.argtypes = [ctypes.c_char_p, i, vp]
        L.kb200_free.argtypes = [vp]
        L.kb200_free.restype = None
        L.kb200_io_error.restype = ctypes.c_char_p
        L.kb200_io_error.argtypes = []
        L.kb200_kaffpa_batch.argtypes = [ctypes.POINTER(BatchItem), i, i, ctypes.POINTER(BatchReport)]
        L.kb200_kaffpa_population.argtypes = [i, vp, vp, vp, vp, i, d, i, vp, i, vp, vp, i,
                                              ctypes.POINTER(BatchReport)]
        L.kb200_lp_cluster.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), i, vp]
        L.kb200_contract.argtypes = [i, vp, vp, vp, vp, vp, c_int_p, c_ll_p, vp, vp, vp, vp, vp]
        L.kb200_lp_refine.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), i, u32, vp]
        L.kb200_jet_refine.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), i, u32, vp]
        L.kb200_balance.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), i, u32, vp, c_int_p]
        L.kb200_edge_cut.argtypes = [i, vp, vp, vp, vp, vp, i, c_ll_p, vp]
        L.kb200_project.argtypes = [i, vp, i, vp, vp]
        L.kb200_initial_partition.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), vp]
        L.kb200_initial_partition_device.argtypes = [i, vp, vp, vp, vp, ctypes.POINTER(Knobs), vp]
        L.kb200_last_error.restype = ctypes.c_char_p
        L.kb200_last_error.argtypes = []
        L.kb200_device_count.argtypes = []
        L.kb200_kernel_launches.argtypes = []
        L.kb200_kernel_launches.restype = ctypes.c_longlong
        L.kaffpa.argtypes = [c_int_p, vp, vp, vp, vp, c_int_p, ctypes.POINTER(d), ctypes.c_bool, i, i,
                             c_int_p, vp]
        L.kaffpa.restype = None
        L.kaffpa_balance.argtypes = [c_int_p, vp, vp, vp, vp, c_int_p, ctypes.POINTER(d), ctypes.c_bool,
                                     ctypes.c_bool, i, i, c_int_p, vp]
        L.kaffpa_balance.restype = None
        _LIB = L
    return _LIB


class KaHIPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"kb200 status {code}: {msg}")
        self.code = code


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def _check(rc: int):
    if rc < 0:
        raise KaHIPError(rc, lib().kb200_last_error().decode())
    return rc


def derive_knobs(n: int, vwgt, k: int, imbalance=0.03, seed=0, mode=FAST) -> Knobs:
    kn = Knobs()
    vw = _i32(vwgt)
    _check(lib().kb200_derive_knobs(n, _ptr(vw), k, imbalance, seed, mode, ctypes.byref(kn)))
    return kn


def kaffpa_ex(xadj, adjncy, nparts, imbalance=0.03, seed=0, mode=FAST, vwgt=None, adjwgt=None,
              stats: Stats | None = None):
    """Returns (status, edgecut, part)."""
    xadj, adjncy, vwgt, adjwgt = _i32(xadj), _i32(adjncy), _i32(vwgt), _i32(adjwgt)
    n = len(xadj) - 1
    part = np.zeros(max(n, 0), np.int32)
    cut = ctypes.c_longlong(-1)
    rc = lib().kb200_kaffpa(n, _ptr(vwgt), _ptr(xadj), _ptr(adjwgt), _ptr(adjncy), nparts, imbalance, seed,
                            mode, ctypes.byref(cut), _ptr(part), ctypes.byref(stats) if stats else None)
    _check(rc)
    return rc, cut.value, part


def kaffpa_knobs(xadj, adjncy, kn: Knobs, vwgt=None, adjwgt=None, stats: Stats | None = None):
    """Whole partitioning with explicit knobs.  Returns (status, edgecut, part)."""
    xadj, adjncy, vwgt, adjwgt = _i32(xadj), _i32(adjncy), _i32(vwgt), _i32(adjwgt)
    n = len(xadj) - 1
    part = np.zeros(max(n, 0), np.int32)
    cut = ctypes.c_longlong(-1)
    rc = lib().kb200_kaffpa_knobs(n, _ptr(vwgt), _ptr(xadj), _ptr(adjwgt), _ptr(adjncy), ctypes.byref(kn),
                                  ctypes.byref(cut), _ptr(part), ctypes.byref(stats) if stats else None)
    _check(rc)
    return rc, cut.value, part


def kaffpa_combine(g: dict, kn: Knobs, part_a, part_b, stats: Stats | None = None, unit_weights=False):
    """KaFFPaE combine of two partitions of g (kb200_kaffpa_combine).
    Returns (status, edgecut, part)."""
    n = g["n"]
    xadj, adjncy = _i32(g["xadj"]), _i32(g["adjncy"])
    vwgt = None if unit_weights else _i32(g["vwgt"])
    adjwgt = None if unit_weights else _i32(g["adjwgt"])
    pa = np.ascontiguousarray(part_a, dtype=np.int32)
    pb = np.ascontiguousarray(part_b, dtype=np.int32)
    part = np.zeros(max(n, 0), np.int32)
    cut = ctypes.c_longlong(-1)
    rc = lib().kb200_kaffpa_combine(n, _ptr(vwgt), _ptr(xadj), _ptr(adjwgt), _ptr(adjncy), ctypes.byref(kn),
                                    _ptr(pa), _ptr(pb), ctypes.byref(cut), _ptr(part),
                                    ctypes.byref(stats) if stats else None)
    _check(rc)
    return rc, cut.value, part


def kaffpae(g: dict, kn: Knobs, population: int, generations: int, per_generation: int, workers=0,
            unit_weights=False):
    """KaFFPaE-style evolution on the device (kb200_kaffpae).
    Returns (status, edgecut, part, history)."""
    n = g["n"]
    xadj, adjncy = _i32(g["xadj"]), _i32(g["adjncy"])
    vwgt = None if unit_weights else _i32(g["vwgt"])
    adjwgt = None if unit_weights else _i32(g["adjwgt"])
    part = np.zeros(max(n, 0), np.int32)
    hist = np.zeros(max(generations, 0) + 1, np.int64)
    cut = ctypes.c_longlong(-1)
    rc = lib().kb200_kaffpae(n, _ptr(vwgt), _ptr(xadj), _ptr(adjwgt), _ptr(adjncy), ctypes.byref(kn), population,
                             generations, per_generation, workers, ctypes.byref(cut), _ptr(part), hist.ctypes.data)
    _check(rc)
    return rc, cut.value, part, hist


def hem_match(g: dict, kn: Knobs, level=0, rating=None) -> np.ndarray:
    """Heavy-edge matching labels of one level; rating: optional uint32 per directed entry."""
    lab = np.empty(g["n"], np.int32)
    rq = None if rating is None else np.ascontiguousarray(rating, np.uint32)
    _check(lib().kb200_hem_match(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]),
                                 _ptr(g["vwgt"]), ctypes.byref(kn), level,
                                 None if rq is None else rq.ctypes.data_as(ctypes.c_void_p), _ptr(lab)))
    return lab


def lp_cluster(g: dict, kn: Knobs, level=0) -> np.ndarray:
    lab = np.empty(g["n"], np.int32)
    _check(lib().kb200_lp_cluster(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]),
                                  _ptr(g["vwgt"]), ctypes.byref(kn), level, _ptr(lab)))
    return lab


def contract(g: dict, label):
    n, m = g["n"], g["m"]
    nc, mc = ctypes.c_int(), ctypes.c_longlong()
    cmap = np.empty(n, np.int32)
    cx = np.empty(n + 1, np.int32)
    ca = np.empty(max(m, 1), np.int32)
    cw = np.empty(max(m, 1), np.int32)
    cv = np.empty(max(n, 1), np.int32)
    lab = _i32(label)
    _check(lib().kb200_contract(n, _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]), _ptr(g["vwgt"]),
                                _ptr(lab), ctypes.byref(nc), ctypes.byref(mc), _ptr(cmap), _ptr(cx), _ptr(ca),
                                _ptr(cw), _ptr(cv)))
    k, mk = nc.value, mc.value
    return dict(n=k, m=mk, xadj=cx[:k + 1].copy(), adjncy=ca[:mk].copy(), adjwgt=cw[:mk].copy(),
                vwgt=cv[:k].copy()), cmap


def jet_refine(g: dict, kn: Knobs, part, bound: int, level=0) -> np.ndarray:
    p = np.array(part, np.int32)
    _check(lib().kb200_jet_refine(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]),
                                  _ptr(g["vwgt"]), ctypes.byref(kn), level, bound, _ptr(p)))
    return p


def lp_refine(g: dict, kn: Knobs, part, bound: int, level=0) -> np.ndarray:
    p = np.array(part, np.int32)
    _check(lib().kb200_lp_refine(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]),
                                 _ptr(g["vwgt"]), ctypes.byref(kn), level, bound, _ptr(p)))
    return p


def balance(g: dict, kn: Knobs, part, bound: int, level=0):
    p = np.array(part, np.int32)
    ok = ctypes.c_int(0)
    _check(lib().kb200_balance(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]), _ptr(g["vwgt"]),
                               ctypes.byref(kn), level, bound, _ptr(p), ctypes.byref(ok)))
    return p, ok.value


def edge_cut(g: dict, part, k: int):
    """Returns (cut, block_weights)."""
    cut = ctypes.c_longlong()
    bw = np.zeros(k, np.uint32)
    p = _i32(part)
    _check(lib().kb200_edge_cut(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]), _ptr(g["vwgt"]),
                                _ptr(p), k, ctypes.byref(cut), _ptr(bw)))
    return cut.value, bw


def project(cmap, nc: int, part_coarse) -> np.ndarray:
    cm, pc = _i32(cmap), _i32(part_coarse)
    out = np.empty(len(cm), np.int32)
    _check(lib().kb200_project(len(cm), _ptr(cm), nc, _ptr(pc), _ptr(out)))
    return out


def initial_partition(g: dict, kn: Knobs) -> np.ndarray:
    p = np.empty(g["n"], np.int32)
    _check(lib().kb200_initial_partition(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]),
                                         _ptr(g["vwgt"]), ctypes.byref(kn), _ptr(p)))
    return p


def initial_partition_device(g: dict, kn: Knobs) -> np.ndarray:
    """The device initial partitioner (every bisection of a recursion depth
    in one launch) on a host graph."""
    p = np.empty(g["n"], np.int32)
    _check(lib().kb200_initial_partition_device(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]),
                                                _ptr(g["vwgt"]), ctypes.byref(kn), _ptr(p)))
    return p


def device_count() -> int:
    return lib().kb200_device_count()


def kernel_launches() -> int:
    return lib().kb200_kernel_launches()


def kaffpa_device(n, xadj, adjncy, adjwgt, vwgt, part, nparts, imbalance=0.03, seed=0, mode=FAST,
                  stream=None, stats: Stats | None = None):
    """Device-resident call: every array is a CUDA tensor (int32) of the current
    device; stream is a torch.cuda.Stream (or None).  Returns (status, edgecut)."""
    cut = ctypes.c_longlong(-1)
    rc = lib().kb200_kaffpa_device(n, _ptr(vwgt), _ptr(xadj), _ptr(adjwgt), _ptr(adjncy), nparts, imbalance,
                                   seed, mode, ctypes.byref(cut), _ptr(part),
                                   None if stream is None else stream.cuda_stream,
                                   ctypes.byref(stats) if stats else None)
    _check(rc)
    return rc, cut.value


def kaffpa_device_knobs(n, xadj, adjncy, adjwgt, vwgt, part, kn: Knobs, stream=None, stats: Stats | None = None):
    """kaffpa_device with explicit knobs (kn.k blocks).  Returns (status, edgecut)."""
    cut = ctypes.c_longlong(-1)
    rc = lib().kb200_kaffpa_device_knobs(n, _ptr(vwgt), _ptr(xadj), _ptr(adjwgt), _ptr(adjncy), ctypes.byref(kn),
                                         ctypes.byref(cut), _ptr(part),
                                         None if stream is None else stream.cuda_stream,
                                         ctypes.byref(stats) if stats else None)
    _check(rc)
    return rc, cut.value


def kaffpa_batch(graphs: list, nparts, imbalance=0.03, seeds=0, modes=FAST, workers=0):
    """Partitions many host graphs (dicts with xadj/adjncy and optional
    adjwgt/vwgt) in one batch.  nparts/imbalance/seeds/modes: scalars or one
    per graph.  Returns (cuts, parts, statuses, report)."""
    cnt = len(graphs)

    def per(x):
        return list(x) if isinstance(x, (list, tuple, np.ndarray)) else [x] * cnt

    ks, imbs, sds, mds = per(nparts), per(imbalance), per(seeds), per(modes)
    keep = []
    items = (BatchItem * max(cnt, 1))()
    parts = []
    for i, g in enumerate(graphs):
        arrs = [_i32(g.get(key)) for key in ("xadj", "adjncy", "adjwgt", "vwgt")]
        keep.append(arrs)
        n = len(arrs[0]) - 1
        p = np.zeros(max(n, 0), np.int32)
        parts.append(p)
        items[i] = BatchItem(n, _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), _ptr(arrs[3]), int(ks[i]),
                             float(imbs[i]), int(sds[i]), int(mds[i]), _ptr(p), -1, 0)
    rep = BatchReport()
    rc = lib().kb200_kaffpa_batch(items, cnt, workers, ctypes.byref(rep))
    cuts = np.array([items[i].edgecut for i in range(cnt)], np.int64)
    status = np.array([items[i].status for i in range(cnt)], np.int32)
    if rc < 0 and rep.failed == 0:
        _check(rc)
    return cuts, parts, status, rep


def kaffpa_population(n, xadj, adjncy, adjwgt, vwgt, parts, nparts, seeds, imbalance=0.03, mode=FAST, workers=0):
    """One device-resident graph (CUDA int32 tensors), len(seeds) members;
    parts: CUDA int32 tensor of len(seeds) * n.  Returns (cuts, report)."""
    sd = np.ascontiguousarray(seeds, np.int32)
    cuts = np.full(len(sd), -1, np.int64)
    rep = BatchReport()
    _check(lib().kb200_kaffpa_population(n, _ptr(vwgt), _ptr(xadj), _ptr(adjwgt), _ptr(adjncy), nparts, imbalance,
                                         mode, _ptr(sd), len(sd), _ptr(cuts), _ptr(parts), workers,
                                         ctypes.byref(rep)))
    return cuts, rep


# ------------------------------------------------------ learned edge rating

def rating_infer(g: dict, params, use_tc=True):
    """(prob[m] float32, rating[m] uint32) of every directed entry of g."""
    P = np.ascontiguousarray(params, np.float32)
    assert P.size == RATING_PARAMS
    m = int(g["xadj"][-1])
    prob = np.empty(max(m, 1), np.float32)
    rat = np.empty(max(m, 1), np.uint32)
    _check(lib().kb200_rating_infer(g["n"], _ptr(g["xadj"]), _ptr(g["adjncy"]), _ptr(g["adjwgt"]), _ptr(g["vwgt"]),
                                    _ptr(P), 1 if use_tc else 0, _ptr(prob), _ptr(rat)))
    return prob[:m], rat[:m]


def _train_structs(graphs_labels):
    keep = []
    arr = (TrainGraph * len(graphs_labels))()
    for i, (g, lab) in enumerate(graphs_labels):
        a = [_i32(g[k]) for k in ("xadj", "adjncy", "adjwgt", "vwgt")]
        lb = np.ascontiguousarray(lab, np.uint8)
        keep.append((a, lb))
        arr[i] = TrainGraph(g["n"], _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), _ptr(a[3]), _ptr(lb))
    return arr, keep


def rating_train(graphs_labels, params, steps: int, lr=3e-3):
    """Trains in place on [(graph, label[m]), ...]; returns (params, loss[steps])."""
    P = np.array(params, np.float32, copy=True)
    arr, keep = _train_structs(graphs_labels)
    loss = np.zeros(max(steps, 1), np.float32)
    _check(lib().kb200_rating_train(arr, len(graphs_labels), steps, ctypes.c_float(lr), _ptr(P), _ptr(loss)))
    return P, loss[:steps]


def rating_grad(g: dict, label, params):
    """(grad[RATING_PARAMS], loss) of one graph."""
    P = np.ascontiguousarray(params, np.float32)
    arr, keep = _train_structs([(g, label)])
    G = np.zeros(RATING_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    _check(lib().kb200_rating_grad(arr, _ptr(P), _ptr(G), _ptr(loss)))
    return G, float(loss[0])


# ------------------------------------------------------------------ files

def _read(fn, path: str) -> dict:
    n, m = ctypes.c_int(), ctypes.c_longlong()
    ptrs = [ctypes.c_void_p() for _ in range(4)]
    rc = fn(os.fsencode(path), ctypes.byref(n), ctypes.byref(m), *[ctypes.byref(p) for p in ptrs])
    if rc < 0:
        raise KaHIPError(rc, lib().kb200_io_error().decode())
    try:
        def arr(p, cnt):
            return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_int)), shape=(max(cnt, 1),))[:cnt].copy()
        N, M = n.value, m.value
        return dict(n=N, m=M, xadj=arr(ptrs[0], N + 1), adjncy=arr(ptrs[1], M), adjwgt=arr(ptrs[2], M),
                    vwgt=arr(ptrs[3], N))
    finally:
        for p in ptrs:
            lib().kb200_free(p)


def read_metis(path: str) -> dict:
    """A METIS text graph file (unit weights filled in)."""
    return _read(lib().kb200_read_metis, path)


def read_bgf(path: str) -> dict:
    """A ParHIP binary graph file (version 3)."""
    return _read(lib().kb200_read_bgf, path)


def write_partition(path: str, part) -> None:
    """One block id per line."""
    p = _i32(part)
    rc = lib().kb200_write_partition(os.fsencode(path), len(p), _ptr(p))
    if rc < 0:
        raise KaHIPError(rc, lib().kb200_io_error().decode())
