"""Learned edge rating: the CUDA-core forward against a plain PyTorch fp32
restatement (same BF16 roundings), the tensor-core (tcgen05) forward against
the CUDA-core one, the hand-written backward against torch autograd, a short
training run, and the matching / kaffpa paths that consume the rating.

Tolerances: BF16 activations (8 significant bits) are rounded after every
layer, and different FP32 summation orders can move a value across a BF16
rounding boundary, so probabilities agree to |dp| <= 0.05 per entry and
<= 2e-3 on average; gradients to 2 % in norm.
"""
import numpy as np
import pytest

from conftest import tie_free

pytestmark = pytest.mark.gpu

PARAMS = 27137
H, Z = 64, 32


@pytest.fixture(scope="module")
def N():
    from kahip_b200 import native
    assert native.device_count() > 0, "no CUDA device: the learned-rating tests need one"
    return native


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    return oracle


def random_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    P = np.zeros(PARAMS, np.float32)
    off = 0

    def put(rows, cols, bias):
        nonlocal off
        P[off:off + rows * cols] = rng.normal(0, scale / np.sqrt(cols), rows * cols)
        off += rows * cols
        if bias:
            P[off:off + rows] = rng.normal(0, 0.1, rows)
            off += rows

    put(H, 2, True)
    for _ in range(3):
        put(H, 2 * H, True)
    put(Z, H, True)
    put(Z, 2, False)
    P[off:off + Z] = rng.normal(0, 1 / np.sqrt(Z), Z)
    off += Z
    P[off] = -1.0
    off += 1
    assert off == PARAMS
    return P


def torch_forward(g, P, st=False):
    """fp32 restatement of the network (see kahip_b200/csrc/learned.cuh);
    st=True makes the BF16 roundings straight-through for autograd."""
    import torch
    if st:
        bf = lambda t: t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()  # noqa: E731
    else:
        bf = lambda t: t.to(torch.bfloat16).to(torch.float32)  # noqa: E731
    n = g["n"]
    xadj = torch.from_numpy(g["xadj"].astype(np.int64))
    adj = torch.from_numpy(g["adjncy"].astype(np.int64))
    w = torch.from_numpy(g["adjwgt"].astype(np.float32))
    vw = g["vwgt"].astype(np.int64)
    deg = (xadj[1:] - xadj[:-1])
    src = torch.repeat_interleave(torch.arange(n), deg)
    Pt = torch.from_numpy(P).clone().requires_grad_(st)
    o = 0

    def take(cnt):
        nonlocal o
        t = Pt[o:o + cnt]
        o += cnt
        return bf(t)

    W0 = take(H * 2).view(H, 2); b0 = take(H)
    Ws = []
    for _ in range(3):
        Ws.append((take(H * 2 * H).view(H, 2 * H), take(H)))
    Wz = take(Z * H).view(Z, H); bz = take(Z)
    Wf = take(Z * 2).view(Z, 2); wo = take(Z); bo = take(1)
    x = torch.stack([torch.log2(1.0 + deg.float()) * 0.125,
                     torch.log2(torch.from_numpy(np.maximum(vw, 1)).float()) * 0.125], 1)
    h = bf(torch.relu(x @ W0.T + b0))
    wd = torch.zeros(n).index_add_(0, src, w)
    inv = torch.where(wd > 0, 1.0 / torch.where(wd > 0, wd, torch.ones_like(wd)), torch.zeros_like(wd))
    for W, b in Ws:
        agg = torch.zeros(n, H).index_add_(0, src, w[:, None] * h[adj])
        agg = bf(agg * inv[:, None])
        h = bf(torch.relu(torch.cat([h, agg], 1) @ W.T + b))
    z = bf(h @ Wz.T + bz)
    den = ((vw[g["adjncy"]] * np.repeat(vw, np.diff(g["xadj"]))) & 0xFFFFFFFF).astype(np.float64)
    wl = g["adjwgt"].astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(den > 0, wl * wl / np.where(den > 0, den, 1), np.inf)
    r = np.minimum(np.nan_to_num(r, nan=1e30, posinf=1e30), 1e30)
    f0 = torch.log2(torch.clamp(w, min=1.0)) * 0.125
    f1 = torch.log2(1.0 + torch.from_numpy(r.astype(np.float32))) * 0.125
    t = z[src] + z[adj] + (f0[:, None] * Wf[:, 0] + f1[:, None] * Wf[:, 1])
    s = bo + torch.relu(t) @ wo
    return s, Pt


def graphs_for_tests(graphs):
    g1 = graphs.rgg2d(3000, seed=1)
    g2 = tie_free(graphs.rmat(11, seed=2))
    g2["adjwgt"] = (g2["adjwgt"] % 7 + 1).astype(np.int32)
    g2["vwgt"] = np.random.default_rng(3).integers(1, 9, g2["n"]).astype(np.int32)
    g3 = graphs.grid2d(40, 37)
    # two hubs of 1500 and 2500 entries (rows longer than the tensor-core
    # kernel's gather limit go through the per-row pre-sum) on a ring
    from conftest import csr_from_edges
    n4 = 4100
    edges = [(v, (v + 1) % n4) for v in range(2, n4)] + [(0, v) for v in range(2, 1502)] + \
            [(1, v) for v in range(1600, 4100)]
    g4 = csr_from_edges(n4, edges, weights=[1 + (i * 7) % 5 for i in range(len(edges))])
    return [g1, g2, g3, g4]


def test_forward_matches_torch_and_tensor_cores(N, graphs):
    import torch
    for i, g in enumerate(graphs_for_tests(graphs)):
        P = random_params(10 + i)
        p_cc, r_cc = N.rating_infer(g, P, use_tc=False)
        p_tc, r_tc = N.rating_infer(g, P, use_tc=True)
        s_ref, _ = torch_forward(g, P)
        p_ref = torch.sigmoid(s_ref).detach().numpy()
        for p in (p_cc, p_tc):
            d = np.abs(p - p_ref)
            assert d.mean() < 2e-3 and d.max() < 5e-2, (i, d.mean(), d.max())
        assert np.abs(p_cc - p_tc).mean() < 2e-3
        # the rating is floor((1 - p) * 2^24) of the returned probability
        q = np.clip(np.floor((1.0 - p_tc.astype(np.float32)) * np.float32(16777216.0)), 0, 16777215)
        assert np.array_equal(r_tc, q.astype(np.uint32))


def test_rating_is_symmetric(N, graphs):
    for i, g in enumerate(graphs_for_tests(graphs)):
        P = random_params(20 + i)
        n = g["n"]
        src = np.repeat(np.arange(n), np.diff(g["xadj"]))
        key_fw = src.astype(np.int64) * n + g["adjncy"]
        key_bw = g["adjncy"].astype(np.int64) * n + src
        order = np.argsort(key_fw)
        rev = order[np.searchsorted(key_fw[order], key_bw)]
        for use_tc in (False, True):
            _, r = N.rating_infer(g, P, use_tc=use_tc)
            assert np.array_equal(r, r[rev])


def test_gradient_matches_autograd(N, graphs):
    import torch
    g = graphs.rgg2d(1500, seed=7)
    P = random_params(5)
    part = np.arange(g["n"]) * 8 // g["n"]
    src = np.repeat(np.arange(g["n"]), np.diff(g["xadj"]))
    label = (part[src] != part[g["adjncy"]]).astype(np.uint8)
    G, loss = N.rating_grad(g, label, P)
    s, Pt = torch_forward(g, P, st=True)
    y = torch.from_numpy(label.astype(np.float32))
    pos = float(label.sum())
    neg = len(label) - pos
    pw = min(50.0, max(1.0, neg / pos))
    om = torch.where(y > 0, torch.tensor(pw), torch.tensor(1.0))
    L = (om * torch.nn.functional.binary_cross_entropy_with_logits(s, y, reduction="none")).sum() / om.sum()
    L.backward()
    ref = Pt.grad.numpy()
    assert abs(loss - L.item()) < 1e-3 * max(1.0, abs(L.item()))
    assert np.linalg.norm(G - ref) <= 2e-2 * np.linalg.norm(ref)


def test_training_lowers_the_loss(N, graphs):
    data = []
    for s in range(3):
        g = graphs.rgg2d(4000, seed=30 + s)
        _, _, part = N.kaffpa_ex(g["xadj"], g["adjncy"], 8, 0.03, s, 1)
        src = np.repeat(np.arange(g["n"]), np.diff(g["xadj"]))
        data.append((g, (part[src] != part[g["adjncy"]]).astype(np.uint8)))
    P0 = random_params(1, scale=0.5)
    P, loss = N.rating_train(data, P0, steps=240, lr=3e-3)
    assert np.isfinite(loss).all()
    # cut edges of a mesh partition are hard to predict from local features:
    # the loss falls from the random start towards the trivial level
    assert loss[-30:].mean() < 0.93 * loss[:6].mean()
    assert not np.array_equal(P, P0)


def test_learned_rating_drives_the_matching(N, O, graphs):
    for i, g in enumerate(graphs_for_tests(graphs)):
        P = random_params(40 + i)
        _, r = N.rating_infer(g, P, use_tc=True)
        kn_o = O.knobs(g, 16, 0.03, i, 0)
        kn_p = N.derive_knobs(g["n"], g["vwgt"], 16, 0.03, i, 0)
        assert np.array_equal(O.hem_match(g, kn_o, 1, r), N.hem_match(g, kn_p, 1, r))


def test_kaffpa_with_learned_rating(N, O, graphs):
    import ctypes
    g = graphs.rgg2d(1 << 14, seed=11)
    P = random_params(99)
    kn = N.derive_knobs(g["n"], g["vwgt"], 16, 0.03, 0, 0)
    # no model: the expansion*^2 matching, bit for bit
    kn.coarsening = 2
    kn.rating_model = None
    _, cut_none, part_none = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn, vwgt=g["vwgt"], adjwgt=g["adjwgt"])
    kn1 = N.derive_knobs(g["n"], g["vwgt"], 16, 0.03, 0, 0)
    kn1.coarsening = 1
    _, cut_plain, part_plain = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn1, vwgt=g["vwgt"], adjwgt=g["adjwgt"])
    assert cut_none == cut_plain and np.array_equal(part_none, part_plain)
    # with a model: deterministic and balanced
    kn.rating_model = P.ctypes.data_as(ctypes.c_void_p)
    _, c1, p1 = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn, vwgt=g["vwgt"], adjwgt=g["adjwgt"])
    _, c2, p2 = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn, vwgt=g["vwgt"], adjwgt=g["adjwgt"])
    assert c1 == c2 and np.array_equal(p1, p2)
    assert np.bincount(p1, minlength=16).max() <= kn.final_bound
    # the guard keeps whichever cuts less (ratio 1.0)
    kn.rating_fallback = 1.0
    st = N.Stats()
    _, c3, p3 = N.kaffpa_knobs(g["xadj"], g["adjncy"], kn, vwgt=g["vwgt"], adjwgt=g["adjwgt"], stats=st)
    assert c3 == min(c1, cut_plain)
    assert st.rating_fallback_used == (1 if c1 > cut_plain else 0)
