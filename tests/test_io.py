"""Graph and partition files (host code, no GPU): METIS text and ParHIP
binary graphs read back bit-exactly, including comments, isolated vertices
and every weight format; malformed files rejected; the partition writer's
format; and, where the reference sources are present, the reference's own
METIS reader on its example graphs."""
import os
import struct

import numpy as np
import pytest

from conftest import tie_free

REF_EXAMPLES = os.path.join(os.environ.get("KAHIP_REFERENCE", "/root/reference"), "examples")


@pytest.fixture(scope="module")
def N():
    from kahip_b200 import native
    return native


def write_metis(path, g, fmt, comments=False):
    n = g["n"]
    with open(path, "w") as f:
        if comments:
            f.write("% a comment before the header\n")
        f.write(f"{n} {g['m'] // 2}" + (f" {fmt}" if fmt else "") + "\n")
        for v in range(n):
            if comments and v % 97 == 0:
                f.write("% comment line\n")
            parts = []
            if fmt in (10, 11):
                parts.append(str(int(g["vwgt"][v])))
            for e in range(g["xadj"][v], g["xadj"][v + 1]):
                parts.append(str(int(g["adjncy"][e]) + 1))
                if fmt in (1, 11):
                    parts.append(str(int(g["adjwgt"][e])))
            f.write(" ".join(parts) + "\n")


def write_bgf(path, g):
    n, m = g["n"], g["m"]
    base = (3 + n + 1) * 8
    with open(path, "wb") as f:
        f.write(struct.pack("<3Q", 3, n, m))
        f.write((base + 8 * g["xadj"].astype(np.uint64)).astype("<u8").tobytes())
        f.write(g["adjncy"].astype("<u8").tobytes())


def same(a, b, weights=True):
    assert a["n"] == b["n"] and a["m"] == b["m"]
    keys = ("xadj", "adjncy", "adjwgt", "vwgt") if weights else ("xadj", "adjncy")
    for k in keys:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


@pytest.mark.parametrize("fmt", [0, 1, 10, 11])
def test_metis_round_trip(N, graphs, tmp_path, fmt):
    g = tie_free(graphs.rgg2d(3000, seed=fmt))
    g["vwgt"] = np.random.default_rng(fmt).integers(1, 50, g["n"]).astype(np.int32)
    # isolated vertices (empty lines) at both ends and in the middle
    from kahip_b200.graphs import from_csr
    n = g["n"] + 3
    deg = np.concatenate([[0], np.diff(g["xadj"])[:1500], [0], np.diff(g["xadj"])[1500:], [0]])
    remap = np.concatenate([[1 + v for v in range(1500)], [2 + v for v in range(1500, g["n"])]])
    x = np.concatenate([[0], np.cumsum(deg)]).astype(np.int32)
    h = from_csr(x, remap[g["adjncy"]].astype(np.int32), g["adjwgt"],
                 np.concatenate([[5], g["vwgt"][:1500], [6], g["vwgt"][1500:], [7]]).astype(np.int32))
    p = str(tmp_path / "g.graph")
    write_metis(p, h, fmt, comments=True)
    r = N.read_metis(p)
    exp = dict(h)
    if fmt in (0, 10):
        exp["adjwgt"] = np.ones(h["m"], np.int32)
    if fmt in (0, 1):
        exp["vwgt"] = np.ones(n, np.int32)
    same(r, exp)


def test_large_metis_file_parallel_parse(N, graphs, tmp_path):
    g = graphs.rgg2d(1 << 17, seed=3)
    p = str(tmp_path / "big.graph")
    write_metis(p, g, 0)
    same(N.read_metis(p), g)


def test_bgf_round_trip(N, graphs, tmp_path):
    g = graphs.rmat(12, seed=1)
    p = str(tmp_path / "g.bgf")
    write_bgf(p, g)
    r = N.read_bgf(p)
    same(r, g, weights=False)
    assert (r["adjwgt"] == 1).all() and (r["vwgt"] == 1).all()


@pytest.mark.parametrize("text,why", [
    ("3 2\n2\n1 3\n2\n", None),
    ("3 2\n2\n1 3\n", "nodes"),
    ("3 3\n2\n1 3\n2\n", "edges"),
    ("3 2\n2\n1 3 3\n2\n", "edges"),
    ("3 1\n1\n\n\n", "self"),
    ("3 2\n2\n1 4\n2\n", "range"),
    ("3 2 7\n2\n1 3\n2\n", "format"),
    ("x y\n", "header"),
])
def test_metis_errors(N, tmp_path, text, why):
    p = str(tmp_path / "e.graph")
    with open(p, "w") as f:
        f.write(text)
    if why is None:
        g = N.read_metis(p)
        assert g["xadj"].tolist() == [0, 1, 3, 4] and g["adjncy"].tolist() == [1, 0, 2, 1]
        return
    with pytest.raises(N.KaHIPError):
        N.read_metis(p)


def test_write_partition(N, tmp_path):
    part = np.array([0, 7, 12, 3, 255, 0, 100000], np.int32)
    p = str(tmp_path / "part")
    N.write_partition(p, part)
    assert open(p).read() == "".join(f"{x}\n" for x in part)
    N.write_partition(p, np.zeros(0, np.int32))
    assert open(p).read() == ""


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference sources absent")
def test_reference_examples_read_like_the_reference(N):
    from oracle import oracle as O
    for name in ("rgg_n_2_15_s0.graph", "delaunay_n15.graph", "example_weighted.graph"):
        path = os.path.join(REF_EXAMPLES, name)
        mine = N.read_metis(path)
        if O.ref_available():
            same(mine, O.ref_read_metis(path))
    same(N.read_bgf(os.path.join(REF_EXAMPLES, "rgg_n_2_15_s0.bgf")),
         N.read_metis(os.path.join(REF_EXAMPLES, "rgg_n_2_15_s0.graph")), weights=False)
