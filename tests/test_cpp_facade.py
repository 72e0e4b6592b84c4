"""The C++ facade include/panns_searching.hpp: a driver written like the
reference's apps compiles and links against it and libpanns_b200.so (CPU), and
on a GPU reproduces the reference's ids for a golden case (per-query and
batched forms)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_ids

EXE = os.path.join(ROOT, "tests", "cpp", "_facade_driver")


def build_driver():
    from parallel_anns_b200 import build as b
    so = b.build()
    src = os.path.join(ROOT, "tests", "cpp", "facade_driver.cpp")
    cmd = ["/usr/bin/g++", "-O2", "-std=c++14", "-I", os.path.join(ROOT, "include"), src, "-o", EXE,
           "-L", os.path.dirname(so), "-lpanns_b200", f"-Wl,-rpath,{os.path.dirname(so)}"]
    subprocess.run(cmd, check=True)
    return EXE


def test_facade_driver_compiles_and_links():
    exe = build_driver()
    assert os.path.exists(exe)


@pytest.mark.gpu
@pytest.mark.parametrize("form,T,X", [("pss_t1_L100", 1, 1)])
def test_facade_driver_reproduces_reference(form, T, X, golden_manifest):
    exe = build_driver()
    d = os.path.join(GOLDEN, "mix3k_d96")
    spec = golden_manifest["mix3k_d96"]["forms"][form]
    K, L = spec["args"]["K"], spec["args"]["L"]
    r = subprocess.run([exe, os.path.join(d, "base.fvecs"), os.path.join(d, "query.fvecs"),
                        os.path.join(d, "graph.nsg"), str(K), str(L), str(T), str(X)],
                       capture_output=True, text=True, check=True)
    ids = np.array([[int(x) for x in line.split()] for line in r.stdout.strip().splitlines()], np.uint32)
    assert np.array_equal(ids, golden_ids("mix3k_d96", form, K))
    assert "batch_equal=1" in r.stderr
