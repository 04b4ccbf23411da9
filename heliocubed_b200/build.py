"""Build the product library heliocubed_b200/libhc_b200.so for sm_100a.

nvcc -gencode arch=compute_100a,code=sm_100a on every CUDA translation unit,
host C++ compiled by nvcc's host compiler, linked into one shared library
with the C ABI of include/hc_abi.h.  Objects go to heliocubed_b200/_build/.

Run: python -m heliocubed_b200.build [--force]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", os.path.join(REPO, "include")]
SOURCES = ["hc_kernels.cu", "hc_context.cpp", "hc_noalloc.cu", "hc_o4.cu", "hc_o4level.cu", "hc_cme.cu", "hc_amr.cu"]
HEADERS = ["hc_device.cuh", "hc_level.h", "hc_common.h"]


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the stale translation units (in parallel, one nvcc process
    each) and link the library."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(REPO, "include", "hc_abi.h")]
    objs, cmds = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path, *headers, __file__]):
            cmd = [NVCC, *ARCH, *COMMON, "-c", path, "-o", obj]
            if src.endswith(".cu") and verbose:
                cmd += ["-Xptxas", "-v"]
            if src.endswith(".cpp"):
                cmd = [NVCC, *ARCH, *COMMON, "-x", "c++", "-c", path, "-o", obj]
            cmds.append(cmd)
    if cmds:
        with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
            for r in list(pool.map(lambda c: subprocess.run(c), cmds)):
                if r.returncode != 0:
                    raise subprocess.CalledProcessError(r.returncode, r.args)
    if force or _stale(LIB, objs):
        subprocess.run([NVCC, *ARCH, "-shared", "--cudart", "static", *objs, "-o", LIB], check=True)
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
