"""Host-side checks that need no GPU: the C-ABI library builds, loads and
exports every function include/panns_b200.h declares; host-only entry points
(recall, true-NN reader, rand replay) behave like the reference; file formats
round-trip."""
import ctypes
import os
import re
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(panns_[a-z_0-9]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from parallel_anns_b200 import native as N
    lib = N.load()
    decl = declared_functions()
    assert decl, "no declarations found"
    for name in decl:
        assert hasattr(lib, name), name
    assert set(decl) <= set(N.EXPORTS) | set(decl)
    assert lib.panns_version() >> 16 == 1


def test_open_without_gpu_reports_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from parallel_anns_b200 import native as N
    h = ctypes.c_void_p()
    rc = N.load().panns_open(ctypes.byref(h), 0)
    assert rc == -4
    assert N.load().panns_last_error()


def test_recall_definition():
    from parallel_anns_b200.searching import recall
    true = np.arange(100, dtype=np.uint32)[None, :].repeat(2, 0)
    res = true.copy()
    res[1, :50] += 1000
    assert recall(res, true, 100, 100) == pytest.approx(0.75)
    # only the first min(L, 100) results count
    assert recall(res, true, 50, 100) == pytest.approx(0.25)
    assert recall(res[:, :1], true, 100, 1) == pytest.approx(0.5)


def test_true_nn_reader_matches_writer():
    from parallel_anns_b200 import formats as fm
    from parallel_anns_b200 import native as N
    ids = np.random.default_rng(0).integers(0, 1000, (7, 100)).astype(np.uint32)
    d = np.random.default_rng(1).random((7, 100)).astype(np.float32)
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "gt.bin")
        fm.write_true_nn(p, ids, d)
        nq, K = ctypes.c_uint32(), ctypes.c_uint32()
        lib = N.load()
        N.check(lib.panns_load_true_nn(p.encode(), ctypes.byref(nq), ctypes.byref(K), None, None))
        assert (nq.value, K.value) == (7, 100)
        oi = np.empty((7, 100), np.uint32)
        od = np.empty((7, 100), np.float32)
        N.check(lib.panns_load_true_nn(p.encode(), ctypes.byref(nq), ctypes.byref(K), N.ptr(oi), N.ptr(od)))
        assert np.array_equal(oi, ids) and np.array_equal(od, d)
        with open(p, "r+b") as f:
            f.truncate(100)
        rc = lib.panns_load_true_nn(p.encode(), ctypes.byref(nq), ctypes.byref(K), N.ptr(oi), N.ptr(od))
        assert rc == -2


def test_formats_roundtrip():
    from parallel_anns_b200 import formats as fm
    g = fm.read_nsg(os.path.join(GOLDEN, "mix1k_d24", "graph.nsg"))
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "g.nsg")
        fm.write_nsg(p, g)
        assert open(p, "rb").read() == open(os.path.join(GOLDEN, "mix1k_d24", "graph.nsg"), "rb").read()
        x = np.random.default_rng(0).random((5, 16)).astype(np.float32)
        fm.write_fvecs(os.path.join(t, "x.fvecs"), x)
        assert np.array_equal(fm.read_fvecs(os.path.join(t, "x.fvecs")), x)
        r = np.arange(30, dtype=np.uint32).reshape(3, 10)
        fm.write_results(os.path.join(t, "r.bin"), r)
        assert np.array_equal(fm.read_results(os.path.join(t, "r.bin")), r)
