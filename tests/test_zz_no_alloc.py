"""kb200_edge_cut_noalloc: the entry point for callers that must not allocate
device memory (fixed memory budgets, allocator-free sections, memory owned by
another runtime) -- checked against the CPU oracle's edge cut and block
weights and against the allocating kb200_edge_cut.

Runs last (file name) so that a stopped-at-first-failure run has already run
every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import tie_free

pytestmark = pytest.mark.gpu


def _fn(native):
    fn = native.lib().kb200_edge_cut_noalloc
    vp = ctypes.c_void_p
    fn.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp]
    fn.restype = ctypes.c_int
    return fn


def test_noalloc_matches_allocating_entry_point(graphs):
    import torch

    from kahip_b200 import native

    assert native.device_count() > 0, "needs a CUDA device"
    fn = _fn(native)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = tie_free(graphs.rgg2d(1 << 14, seed=3), seed=3)
    rng = np.random.default_rng(11)
    g["vwgt"] = rng.integers(1, 5, g["n"]).astype(np.int32)
    d = {k: torch.from_numpy(np.ascontiguousarray(g[k])).to(dev) for k in ("xadj", "adjncy", "adjwgt", "vwgt")}
    k = 64
    d_cut = torch.zeros(1, dtype=torch.int64, device=dev)
    d_bw = torch.zeros(k, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call(part, kk, bw):
        d_part = torch.from_numpy(part).to(dev)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        rc = fn(g["n"], d["xadj"].data_ptr(), d["adjncy"].data_ptr(), d["adjwgt"].data_ptr(), d["vwgt"].data_ptr(),
                d_part.data_ptr(), kk, d_cut.data_ptr(), bw.data_ptr(), stream)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info(dev)[0]
        assert rc == 0, native.lib().kb200_last_error()
        return free0, free1

    from oracle import oracle

    results = []
    for i in range(3):  # two calls in a row (and a third to watch device memory)
        part = rng.integers(0, k, g["n"]).astype(np.int32)
        free0, free1 = call(part, k, d_bw)
        assert d_cut.item() == oracle.edge_cut(g, part)
        assert np.array_equal(d_bw.cpu().numpy().view(np.uint32), oracle.block_weights(g, part, k))
        cut_ref, bw_ref = native.edge_cut(g, part, k)   # the allocating entry point
        assert d_cut.item() == cut_ref
        assert np.array_equal(d_bw.cpu().numpy().view(np.uint32), bw_ref)
        results.append((free0, free1))
    # after the first call (module load), a call changes no device allocation
    assert results[1][0] == results[1][1] and results[2][0] == results[2][1]

    # a smaller k after a larger one: only its slots are used and cleared
    part = rng.integers(0, 5, g["n"]).astype(np.int32)
    bw5 = torch.zeros(5, dtype=torch.int32, device=dev)
    call(part, 5, bw5)
    cut_ref, bw_ref = native.edge_cut(g, part, 5)
    assert d_cut.item() == cut_ref
    assert np.array_equal(bw5.cpu().numpy().view(np.uint32), bw_ref)

    # limits: k beyond the stated maximum is rejected, out-of-range ids give -1
    rc = fn(g["n"], d["xadj"].data_ptr(), d["adjncy"].data_ptr(), None, None,
            torch.zeros(g["n"], dtype=torch.int32, device=dev).data_ptr(), 65537, d_cut.data_ptr(),
            d_bw.data_ptr(), stream)
    assert rc == native.ERR_INVALID_INPUT
    bad = np.zeros(g["n"], np.int32)
    bad[7] = 9
    call(bad, 4, torch.zeros(4, dtype=torch.int32, device=dev))
    assert d_cut.item() == -1
    # a negative edge weight is refused like the other entry points refuse it
    neg = d["adjwgt"].clone()
    neg[3] = -5
    part = rng.integers(0, 4, g["n"]).astype(np.int32)
    d_part = torch.from_numpy(part).to(dev)
    rc = fn(g["n"], d["xadj"].data_ptr(), d["adjncy"].data_ptr(), neg.data_ptr(), None, d_part.data_ptr(), 4,
            d_cut.data_ptr(), d_bw.data_ptr(), stream)
    torch.cuda.synchronize()
    assert rc == 0 and d_cut.item() == -1
    # and the next valid call is unaffected by the refused ones
    call(part, 4, bw5)
    assert d_cut.item() == oracle.edge_cut(g, part)
