"""Seeded synthetic graphs (int32 METIS-style CSR) from libkb200_graphgen.so.

Graph = dict(n, xadj, adjncy, adjwgt, vwgt) of numpy int32 arrays.  The
generators are deterministic functions of their arguments (counter-based
randomness), so tests, the oracle and the benchmark see identical inputs.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libkb200_graphgen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build() first")
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.kbgen_rgg2d.restype = vp
        L.kbgen_rgg2d.argtypes = [ctypes.c_longlong, ctypes.c_double, ctypes.c_ulonglong]
        L.kbgen_rgg3d.restype = vp
        L.kbgen_rgg3d.argtypes = [ctypes.c_longlong, ctypes.c_double, ctypes.c_ulonglong]
        L.kbgen_rmat.restype = vp
        L.kbgen_rmat.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong]
        L.kbgen_grid2d.restype = vp
        L.kbgen_grid2d.argtypes = [ctypes.c_longlong, ctypes.c_longlong]
        for f in (L.kbgen_n, L.kbgen_m):
            f.restype = ctypes.c_longlong
            f.argtypes = [vp]
        L.kbgen_has_adjwgt.restype = ctypes.c_int
        L.kbgen_has_adjwgt.argtypes = [vp]
        L.kbgen_copy.restype = None
        L.kbgen_copy.argtypes = [vp, vp, vp, vp, vp]
        L.kbgen_free.restype = None
        L.kbgen_free.argtypes = [vp]
        _LIB = L
    return _LIB


def _take(handle, out=None):
    L = _lib()
    if not handle:
        raise ValueError("generator rejected its arguments (or the graph exceeds int32 edges)")
    try:
        n, m = L.kbgen_n(handle), L.kbgen_m(handle)
        if out is None:
            out = dict(xadj=np.empty(n + 1, np.int32), adjncy=np.empty(m, np.int32),
                       adjwgt=np.empty(m, np.int32), vwgt=np.empty(n, np.int32))
        ptr = lambda a: a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr()
        L.kbgen_copy(handle, ptr(out["xadj"]), ptr(out["adjncy"]), ptr(out["adjwgt"]), ptr(out["vwgt"]))
        out["n"] = int(n)
        out["m"] = int(m)
        return out
    finally:
        L.kbgen_free(handle)


def rgg2d(n: int, seed: int = 0, r_factor: float = 0.55) -> dict:
    """2D random geometric graph, radius r_factor*sqrt(ln n / n), unit weights."""
    return _take(_lib().kbgen_rgg2d(n, r_factor, seed))


def rgg3d(n: int, seed: int = 0, r_factor: float = 0.55) -> dict:
    """3D random geometric graph, radius r_factor*cbrt(ln n / n), unit weights."""
    return _take(_lib().kbgen_rgg3d(n, r_factor, seed))


def rmat(scale: int, samples: int | None = None, a=0.57, b=0.19, c=0.19, seed: int = 0) -> dict:
    """R-MAT, 2^scale nodes, `samples` edge samples (default 16n), symmetrised,
    no self loops, duplicate multiplicity as edge weight."""
    if samples is None:
        samples = 16 << scale
    return _take(_lib().kbgen_rmat(scale, samples, a, b, c, seed))


def grid2d(nx: int, ny: int) -> dict:
    """nx x ny grid with the 5-point stencil, unit weights."""
    return _take(_lib().kbgen_grid2d(nx, ny))


def from_csr(xadj, adjncy, adjwgt=None, vwgt=None) -> dict:
    xadj = np.ascontiguousarray(xadj, np.int32)
    adjncy = np.ascontiguousarray(adjncy, np.int32)
    n = len(xadj) - 1
    m = int(xadj[-1])
    return dict(n=n, m=m, xadj=xadj, adjncy=adjncy,
                adjwgt=np.ones(m, np.int32) if adjwgt is None else np.ascontiguousarray(adjwgt, np.int32),
                vwgt=np.ones(n, np.int32) if vwgt is None else np.ascontiguousarray(vwgt, np.int32))


def batch_specs(count: int, seed: int = 0, nmin: float = 1e3, nmax: float = 2e5,
                ks=(2, 4, 8, 16, 32, 64)) -> list:
    """Seeded specs (kind, n, k, graph_seed) of the batched form's graphs: n
    log-uniform in [nmin, nmax], kind uniform over 2D RGG / 2D grid / R-MAT,
    k uniform over `ks`."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        kind = int(rng.integers(0, 3))
        k = int(ks[int(rng.integers(0, len(ks)))])
        gs = int(rng.integers(0, 1 << 30))
        out.append((kind, n, k, gs))
    return out


def batch_graph(spec) -> dict:
    """The graph of one batch spec: RGG2D (r = 0.55 sqrt(ln n / n)), grid with
    the 5-point stencil (nx*ny ~ n) or R-MAT (2^round(log2 n) nodes, 4 samples
    per node -> average degree ~8, a,b,c = .57,.19,.19)."""
    kind, n, _, gs = spec
    if kind == 0:
        return rgg2d(n, seed=gs)
    if kind == 1:
        nx = max(1, int(round(np.sqrt(n))))
        return grid2d(nx, max(1, n // nx))
    scale = max(1, int(round(np.log2(n))))
    return rmat(scale, samples=4 << scale, seed=gs)


def batch_mix(count: int, seed: int = 0, nmin: float = 1e3, nmax: float = 2e5,
              ks=(2, 4, 8, 16, 32, 64)) -> list:
    """A seeded mix of independent graphs for the batched form (see
    batch_specs / batch_graph).  Returns [(graph, k), ...]."""
    return [(batch_graph(sp), sp[2]) for sp in batch_specs(count, seed, nmin, nmax, ks)]
