"""Generate tests/golden/riemann_pin.npz from the reference's own pointwise
solvers (src/MHD_Roe8Wave.H, src/MHD_SecondOrderFlux.H compiled from the
reference tree by oracle/build.py into oracle/_ref/libhcref.so), and
tests/golden/berta_pin.npz from the reference's fourth-order pointwise
kernels (WENOZ/WENO3/PLM face states, stencil normalisation, Jameson flag,
point/average corrections, reconstruction select, mapped-flux line,
f_sphToPrim, f_primflux, mapped and factored Roe, usable-state check; the
inputs are oracle/berta_pin.cases(20261205)).

The fixture pins the oracle's restatement (tests/test_oracle_pin.py) on
machines where the reference tree is absent.  Inputs are seeded random
solar-wind-like primitive states (CGS) in the face frame, including cases
where the Roe fan check falls back to Rusanov.

Run: python tests/golden/make_golden.py
(needs HC_REFERENCE=<reference tree> python oracle/build.py first)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402

C_MP = 1.67262192e-24
BERTA_SEED = 20261205
BERTA_CASES = 256


def states(rng, n):
    s = np.empty((n, 8))
    s[:, 0] = 700 * C_MP * rng.uniform(0.05, 4, n)
    s[:, 1:4] = rng.normal(0, 3e7, (n, 3))
    s[:, 4] = 1e-7 * rng.uniform(0.01, 3, n)
    s[:, 5:8] = rng.normal(0, 1e-4, (n, 3)) * rng.choice([0.0, 1.0], (n, 1))
    return s


def main() -> int:
    R = po.ref_lib()
    if R is None:
        print("reference pin library missing: run python oracle/build.py", file=sys.stderr)
        return 1
    rng = np.random.default_rng(20261203)
    n = 256
    wl = states(rng, n)
    wr = states(rng, n)
    close = rng.random(n) < 0.3
    wr[close] = wl[close] * (1 + rng.normal(0, 1e-3, (close.sum(), 8)))
    normals = rng.normal(0, 1, (n, 3))
    area = rng.uniform(0.5, 3.0, n)
    gamma, ef = 5.0 / 3.0, 0.3
    roe = np.zeros((n, 8)); roe_ok = np.zeros(n, dtype=np.int32)
    roe_nc = np.zeros((n, 8)); roe_nc_ok = np.zeros(n, dtype=np.int32)
    rus = np.zeros((n, 8)); flux_rus = np.zeros((n, 8)); flux_roe = np.zeros((n, 8))
    frames = np.zeros((n, 9)); norms = np.zeros(n)
    for q in range(n):
        a, b, nv = wl[q].copy(), wr[q].copy(), normals[q].copy()
        o = np.zeros(8)
        roe_ok[q] = R.ref_roe8(po.dptr(a), po.dptr(b), gamma, ef, 1, po.dptr(o)); roe[q] = o
        o = np.zeros(8)
        roe_nc_ok[q] = R.ref_roe8(po.dptr(a), po.dptr(b), gamma, ef, 0, po.dptr(o)); roe_nc[q] = o
        o = np.zeros(8); R.ref_rusanov(po.dptr(a), po.dptr(b), gamma, po.dptr(o)); rus[q] = o
        o = np.zeros(8); R.ref_face_flux(po.dptr(a), po.dptr(b), po.dptr(nv), area[q], gamma, ef, 0, po.dptr(o)); flux_rus[q] = o
        o = np.zeros(8); R.ref_face_flux(po.dptr(a), po.dptr(b), po.dptr(nv), area[q], gamma, ef, 1, po.dptr(o)); flux_roe[q] = o
        f = np.zeros(9); nm = np.zeros(1); R.ref_frame(po.dptr(nv), po.dptr(f), po.dptr(nm)); frames[q] = f; norms[q] = nm[0]
    np.savez_compressed(os.path.join(HERE, "riemann_pin.npz"), wl=wl, wr=wr, normals=normals, area=area,
                        gamma=gamma, entropy=ef, roe=roe, roe_ok=roe_ok, roe_nocheck=roe_nc,
                        roe_nocheck_ok=roe_nc_ok, rusanov=rus, flux_rusanov=flux_rus, flux_roe=flux_roe,
                        frames=frames, norms=norms)
    print("wrote riemann_pin.npz;", int((roe_ok == 0).sum()), "Roe fallbacks of", n)
    from oracle import berta_pin
    cases = berta_pin.cases(BERTA_SEED, n=BERTA_CASES)
    outs = berta_pin.evaluate(R, "ref", cases)
    np.savez_compressed(os.path.join(HERE, "berta_pin.npz"), **{f"in_{k}": v for k, v in cases.items()},
                        **{f"out_{k}": v for k, v in outs.items()})
    print("wrote berta_pin.npz;", BERTA_CASES, "cases")
    return 0


if __name__ == "__main__":
    sys.exit(main())
