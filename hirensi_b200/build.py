"""Build recipe of libhirensi_b200.so (nvcc, sm_100a).

The library is built in-tree under hirensi_b200/_build/ so that it is found
next to the package wherever the package is copied.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libhirensi_b200.so")
SOURCES = ["hrn_capi.cu", "hrn_step.cu", "hrn_assemble.cu", "hrn_inv.cu", "hrn_noalloc.cu", "hrn_elem.cu", "hrn_cnn.cu", "hrn_gtile.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "hirensi_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA source for sm_100a and link the shared library."""
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = [os.path.join(OUT_DIR, src.replace(".cu", ".o")) for src in SOURCES]
    cmds = [[NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj] for src, obj in zip(SOURCES, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), file=sys.stderr)
    # the translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for r in pool.map(lambda cmd: subprocess.run(cmd, capture_output=True, text=True), cmds):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args, r.stdout, r.stderr)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
