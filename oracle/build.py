"""Build recipe for the oracle (test infrastructure only).

* oracle/libhc_oracle.so -- the CPU restatement (hc_oracle.cpp), g++ -O3,
  -ffp-contract=off, OpenMP.  Built wherever the package is built and carried
  to the GPU box with the repository snapshot.
* oracle/_ref/libhcref.so -- the reference's own standalone headers
  (src/MHD_Roe8Wave.H, src/MHD_Reconstruction.H, src/MHD_SecondOrderFlux.H,
  src/MHD_CME.H with the headers it includes)
  compiled from the reference tree where it lies, through ref_pin.cpp.  Built
  only when the reference tree is present; the generated Proto_Accel.H is a
  two-line stub of our own (the reference's Proto dependency is absent).

Run: python oracle/build.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
DEFAULT_REFERENCE = "/root/reference"

CXXFLAGS = ["-std=c++17", "-O3", "-fPIC", "-shared", "-ffp-contract=off", "-march=x86-64-v2"]


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _stale(out: str, srcs: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "hc_oracle.cpp")
    hdr = os.path.join(REPO, "include", "hc_abi.h")
    inc = os.path.join(HERE, "hc_oracle_o4.inc")
    out = os.path.join(HERE, "libhc_oracle.so")
    if force or _stale(out, [src, hdr, inc, __file__]):
        _run(["g++", *CXXFLAGS, "-fopenmp", src, "-o", out])
    return out


def build_reference_pin(reference: str = DEFAULT_REFERENCE, force: bool = False) -> str | None:
    refsrc = os.path.join(reference, "src")
    if not os.path.isfile(os.path.join(refsrc, "MHD_Roe8Wave.H")):
        return None
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    stub = os.path.join(outdir, "Proto_Accel.H")
    with open(stub, "w") as f:
        f.write("#pragma once\n#define ACCEL_DECORATION\n")
    src = os.path.join(HERE, "ref_pin.cpp")
    out = os.path.join(outdir, "libhcref.so")
    deps = [src] + [os.path.join(refsrc, h) for h in (
        "MHD_Roe8Wave.H", "MHD_SecondOrderFlux.H", "MHD_Reconstruction.H", "MHD_CME.H", "MHD_ImportedCME.H",
        "MHD_Time.H", "MHD_JSON.H", "MHD_Constants.H")]
    if force or _stale(out, deps):
        # -iquote keeps the stub ahead of any other Proto_Accel.H; the reference
        # headers are compiled where they lie.
        _run(["g++", *CXXFLAGS, "-I", outdir, "-I", refsrc, src, "-o", out])
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build_oracle(a.force))
    print(build_reference_pin(a.reference, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
