"""The C ABI library loads without a GPU, exports every symbol the headers in
include/ declare, and refuses to compute without a device (no CPU path)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in ("kahip_b200.h", "kaHIP_interface.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?[\s\*]+([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                             text, flags=re.M):
            if m.group(1) not in ("if", "defined"):
                names.add(m.group(1))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    from kahip_b200 import native
    L = native.lib()
    declared = _declared_functions()
    assert {"kaffpa", "kb200_kaffpa", "kb200_lp_cluster", "kb200_edge_cut_noalloc"} <= declared
    for name in declared:
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
    assert set(native.EXPORTS) == declared


def test_every_bound_entry_point_declares_its_argument_types():
    # without argtypes ctypes passes Python ints (array addresses) as 32-bit
    # C ints; kb200_edge_cut_noalloc is bound by its own test
    from kahip_b200 import native
    L = native.lib()
    missing = [e for e in native.EXPORTS
               if e.startswith("kb200_") and e != "kb200_edge_cut_noalloc" and getattr(L, e).argtypes is None]
    assert not missing, missing


def test_no_device_no_fallback():
    from kahip_b200 import native
    if native.device_count() > 0:
        pytest.skip("a CUDA device is present")
    g = __import__("kahip_b200.graphs", fromlist=["rgg2d"]).rgg2d(256, seed=0)
    with pytest.raises(native.KaHIPError) as e:
        native.kaffpa_ex(g["xadj"], g["adjncy"], 4)
    assert e.value.code == native.ERR_NO_DEVICE
    # the drop-in entry point reports failure through edgecut = -1
    L = native.lib()
    n, k, imb, cut = ctypes.c_int(g["n"]), ctypes.c_int(4), ctypes.c_double(0.03), ctypes.c_int(0)
    part = np.zeros(g["n"], np.int32)
    L.kaffpa(ctypes.byref(n), None, g["xadj"].ctypes.data, None, g["adjncy"].ctypes.data, ctypes.byref(k),
             ctypes.byref(imb), True, 0, 0, ctypes.byref(cut), part.ctypes.data)
    assert cut.value == -1


def test_host_validation_before_device():
    # what sizes the upload is checked on the host (monotonicity, targets and
    # weights are checked on the device right after the upload)
    from kahip_b200 import native
    with pytest.raises(native.KaHIPError) as e:
        native.kaffpa_ex(np.array([0, 2, -1]), np.array([1, 0]), 2)
    assert e.value.code == native.ERR_INVALID_INPUT
    with pytest.raises(native.KaHIPError) as e:
        native.kaffpa_ex(np.array([1, 2, 3]), np.array([1, 0]), 2)
    assert e.value.code == native.ERR_INVALID_INPUT
    with pytest.raises(native.KaHIPError) as e:
        native.kaffpa_ex(np.array([0, 1, 2]), np.array([1, 0]), 0)
    assert e.value.code == native.ERR_INVALID_INPUT


def test_edge_cut_rejects_null_partition():
    # checked before any device work, so it needs no GPU
    from kahip_b200 import native
    L = native.lib()
    xadj = np.array([0, 1, 2], np.int32)
    adj = np.array([1, 0], np.int32)
    cut = ctypes.c_longlong(5)
    rc = L.kb200_edge_cut(2, xadj.ctypes.data, adj.ctypes.data, None, None, None, 2, ctypes.byref(cut), None)
    assert rc == native.ERR_INVALID_INPUT
    assert b"invalid" in L.kb200_last_error()


def test_unsupported_siblings_report_failure():
    from kahip_b200 import native
    L = native.lib()
    n, k, imb = ctypes.c_int(3), ctypes.c_int(2), ctypes.c_double(0.03)
    cut = ctypes.c_int(7)
    xadj = np.array([0, 1, 2, 2], np.int32)
    adj = np.array([1, 0], np.int32)
    L.kaffpa_balance_NE.restype = None
    L.kaffpa_balance_NE(ctypes.byref(n), None, xadj.ctypes.data, None, adj.ctypes.data, ctypes.byref(k),
                        ctypes.byref(imb), True, 0, 0, ctypes.byref(cut), np.zeros(3, np.int32).ctypes.data)
    assert cut.value == -1


def test_python_interface_mirrors_reference_module():
    import inspect

    import kahip_b200
    params = list(inspect.signature(kahip_b200.kaffpa).parameters)
    assert params == ["vwgt", "xadj", "adjcwgt", "adjncy", "nparts", "imbalance", "suppress_output", "seed", "mode"]
    g = kahip_b200.kahip_graph()
    g.set_num_nodes(3)
    g.add_undirected_edge(0, 1, 2)
    g.add_undirected_edge(1, 2)
    vwgt, xadj, adjcwgt, adjncy = g.get_csr_arrays()
    assert xadj == [0, 1, 3, 4] and adjncy == [1, 0, 2, 1] and adjcwgt == [2, 2, 1, 1] and vwgt == [1, 1, 1]
