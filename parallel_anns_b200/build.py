"""Build recipe of the native library: nvcc for sm_100a, in-tree.

``python -m parallel_anns_b200.build`` (or ``build()``) compiles
``csrc/*.cu`` into ``parallel_anns_b200/libpanns_b200.so``, which exports the
C ABI declared in ``include/panns_b200.h``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
SO = os.path.join(PKG, "libpanns_b200.so")
SOURCES = [os.path.join(PKG, "csrc", f) for f in
           ("panns_abi.cu", "search_kernels_fp32_ip.cu", "search_kernels_fp32_l2.cu",
            "search_kernels_bf16.cu", "search_kernels_fp8.cu", "pss_kernels.cu", "learned.cu", "graph_build.cu", "search_block_kernels_fp32.cu", "search_block_kernels_bf16.cu",
            "search_block_kernels_fp8.cu", "nsg_build.cu", "tc_screen.cu")]
DEPS = SOURCES + [os.path.join(PKG, "csrc", f) for f in
                  ("search_kernel.cuh", "pss_kernel.cuh", "gt_kernel.cuh", "kernels.h", "search_kernels.inc",
                   "mlp_infer.cuh", "learned.h", "block_kernel.cuh", "graph_types.h", "tc_screen.h")] + [
    os.path.join(ROOT, "include", "panns_b200.h"), os.path.join(ROOT, "include", "panns_learned.h"),
    os.path.join(ROOT, "include", "panns_build.h"),
]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date() -> bool:
    if not os.path.exists(SO):
        return False
    t = os.path.getmtime(SO)
    return all(os.path.getmtime(p) <= t for p in DEPS if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, extra=None, out: str | None = None,
          objdir: str | None = None) -> str:
    """Compile every source to an object in parallel, then link the shared
    library (``out``, default the in-tree library; ``objdir`` for the objects)."""
    so = out or SO
    if not force and out is None and up_to_date():
        return SO
    objdir = objdir or os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs = []
    objs = []
    # An object is reused when it is newer than its source and every shared
    # header, and was built with the same flags (recorded beside it).
    headers = [p for p in DEPS if p not in SOURCES and os.path.exists(p)]
    newest_header = max((os.path.getmtime(p) for p in headers), default=0.0)
    flags_key = " ".join(NVCC_FLAGS + (extra or []))
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        stamp = obj + ".flags"
        if (os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == flags_key
                and os.path.getmtime(obj) > max(os.path.getmtime(src), newest_header)):
            continue
        with open(stamp, "w") as f:
            f.write(flags_key)
        cmd = [nvcc()] + NVCC_FLAGS + (extra or []) + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((cmd, subprocess.Popen(cmd, cwd=PKG)))
    for cmd, p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", so + ".tmp"] + objs + [
        "-lcudart", "-lcublas"]
    subprocess.run(link, check=True, cwd=PKG)
    os.replace(so + ".tmp", so)
    return so


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    extra += [a for a in sys.argv[1:] if a.startswith("-D")]
    out = next((a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--out=")), None)
    objdir = (out + ".objs") if out else None
    print(build(force=True, verbose=v, extra=extra or None, out=out, objdir=objdir))
