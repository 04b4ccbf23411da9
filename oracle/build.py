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
  The reference's fourth-order pointwise kernels live in files whose other
  functions need Proto's BoxData, so the recipe reads the named free
  functions (the WENOZ/WENO3/PLM face kernels, the stencil normalisation,
  the Jameson flag, the point/average corrections, the reconstruction
  select, the mapped-flux line, f_sphToPrim and f_primflux) out of
  src/BoxOp_BertaCubedSphereImplem.H and src/BoxOp_EulerCubedSphere.H at
  build time into oracle/_ref/berta_kernels.inc (git-ignored, never
  committed) and compiles them unchanged through ref_pin_berta.cpp, which
  supplies a stub of Proto's Var accessor and kernel macros.

The reference tree is taken from --reference or the HC_REFERENCE environment
variable; without either, only the oracle is built.

Run: python oracle/build.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)

# Portable ISA for the library that ships with the repository (x86-64-v3:
# AVX2 and FMA instructions; -ffp-contract=off keeps a*b+c unfused, so the
# results do not depend on the ISA).  The timed CPU baseline builds its own
# -march=native copy on the machine that runs it (build_oracle_native).
CXXFLAGS = ["-std=c++17", "-O3", "-fPIC", "-shared", "-ffp-contract=off"]
PORTABLE = ["-march=x86-64-v3"]

# Free functions read out of the reference's fourth-order files: (file, name).
BERTA_KERNELS = [
    ("BoxOp_EulerCubedSphere.H", "f_sphToPrim_F"),
    ("BoxOp_EulerCubedSphere.H", "f_primflux_F"),
    ("BoxOp_BertaCubedSphereImplem.H", "bertaMappedLine"),
    ("BoxOp_BertaCubedSphereImplem.H", "f_berta_jameson_theta_rawF"),
    ("BoxOp_BertaCubedSphereImplem.H", "f_berta_avg_to_point_thetaF"),
    ("BoxOp_BertaCubedSphereImplem.H", "bertaNormalizeWenoStencil"),
    ("BoxOp_BertaCubedSphereImplem.H", "f_wenoz_pointwise_faceF"),
    ("BoxOp_BertaCubedSphereImplem.H", "f_weno3_pointwise_faceF"),
    ("BoxOp_BertaCubedSphereImplem.H", "berta_minmod3_scalar"),
    ("BoxOp_BertaCubedSphereImplem.H", "f_plm_pointwise_faceF"),
    ("BoxOp_BertaCubedSphereImplem.H", "f_select_reconstructionF"),
    ("BoxOp_BertaCubedSphereImplem.H", "f_flux_point_to_avg_thetaF"),
]


def default_reference() -> str | None:
    return os.environ.get("HC_REFERENCE")


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _stale(out: str, srcs: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def _oracle_sources() -> list[str]:
    return [os.path.join(HERE, "hc_oracle.cpp"), os.path.join(REPO, "include", "hc_abi.h"),
            os.path.join(HERE, "hc_oracle_o4.inc"), __file__]


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "hc_oracle.cpp")
    out = os.path.join(HERE, "libhc_oracle.so")
    if force or _stale(out, _oracle_sources()):
        _run(["g++", *CXXFLAGS, *PORTABLE, "-fopenmp", src, "-o", out])
    return out


def _cpu_key() -> str:
    """Short hash of this CPU's model name and feature flags."""
    import hashlib
    text = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    text += line
                if line.strip() == "":
                    break
    except OSError:
        pass
    return hashlib.sha256(text.encode()).hexdigest()[:12]


def build_oracle_native(outdir: str) -> str | None:
    """A -march=native copy of the oracle for the machine that runs it (the
    timed CPU baseline), or None where g++ fails.  Results are the same as
    the portable library's: floating-point contraction stays off."""
    src = os.path.join(HERE, "hc_oracle.cpp")
    outdir = os.path.join(outdir, _cpu_key())  # a build for one CPU model only
    os.makedirs(outdir, exist_ok=True)
    out = os.path.join(outdir, "libhc_oracle_native.so")
    if _stale(out, _oracle_sources()):
        try:
            _run(["g++", *CXXFLAGS, "-march=native", "-fopenmp", src, "-o", out])
        except (subprocess.CalledProcessError, OSError):
            return None
    return out


def _block_end(lines: list[str], start: int, name: str) -> int:
    """Index of the last line of the function whose signature starts at
    `start`: its PROTO_KERNEL_END line for a kernel, else the line that
    closes its outermost brace."""
    for q in range(start, len(lines)):
        if lines[q].lstrip().startswith(f"PROTO_KERNEL_END({name}"):
            return q
        if lines[q].startswith("template") and q > start:
            break
    depth, opened = 0, False
    for q in range(start, len(lines)):
        code = lines[q].split("//", 1)[0]
        for ch in code:
            if ch == "{":
                depth, opened = depth + 1, True
            elif ch == "}":
                depth -= 1
        if opened and depth == 0:
            return q
    raise ValueError(f"end of {name} not found")


def extract_reference_kernels(refsrc: str, out: str) -> None:
    """Write the text of BERTA_KERNELS, in file order, to `out`, each
    preceded by a line comment naming its reference file and lines."""
    pieces = []
    for fname, name in BERTA_KERNELS:
        lines = open(os.path.join(refsrc, fname)).read().split("\n")
        head = re.compile(rf"^\s*(inline\s+)?(ACCEL_DECORATION\s+)?(void|T)\s+{name}\s*(\(|$)")
        sig = next(q for q, ln in enumerate(lines) if head.match(ln))
        first = next(q for q in range(sig, max(sig - 4, -1), -1) if lines[q].startswith("template"))
        last = _block_end(lines, sig, name)
        pieces.append((fname, first, f"// src/{fname}:{first + 1}-{last + 1}\n" + "\n".join(lines[first:last + 1])))
    # RHO00 as the reference defines it
    rho = next(ln for ln in open(os.path.join(refsrc, "BoxOp_EulerCubedSphere.H")).read().split("\n")
               if ln.startswith("#define RHO00"))
    text = ["// Generated by oracle/build.py from the reference tree; not committed.", rho]
    text += [p[2] for p in pieces]
    with open(out, "w") as f:
        f.write("\n\n".join(text) + "\n")


def build_reference_pin(reference: str | None = None, force: bool = False) -> str | None:
    reference = reference or default_reference()
    if not reference:
        return None
    refsrc = os.path.join(reference, "src")
    if not os.path.isfile(os.path.join(refsrc, "MHD_Roe8Wave.H")):
        return None
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    stub = os.path.join(outdir, "Proto_Accel.H")
    with open(stub, "w") as f:
        f.write("#pragma once\n#define ACCEL_DECORATION\n")
    src = os.path.join(HERE, "ref_pin.cpp")
    src_berta = os.path.join(HERE, "ref_pin_berta.cpp")
    out = os.path.join(outdir, "libhcref.so")
    deps = [src, src_berta, __file__] + [os.path.join(refsrc, h) for h in (
        "MHD_Roe8Wave.H", "MHD_SecondOrderFlux.H", "MHD_Reconstruction.H", "MHD_CME.H", "MHD_ImportedCME.H",
        "MHD_Time.H", "MHD_JSON.H", "MHD_Constants.H", "BoxOp_BertaCubedSphereImplem.H",
        "BoxOp_EulerCubedSphere.H")]
    if force or _stale(out, deps):
        extract_reference_kernels(refsrc, os.path.join(outdir, "berta_kernels.inc"))
        # The stub directory comes first so its Proto_Accel.H is the one
        # found; the reference headers are compiled where they lie.
        _run(["g++", *CXXFLAGS, *PORTABLE, "-I", outdir, "-I", refsrc, src, src_berta, "-o", out])
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference tree (default: $HC_REFERENCE)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build_oracle(a.force))
    print(build_reference_pin(a.reference, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
