"""Seeded input cases and evaluation for pinning the oracle's fourth-order
pointwise pieces to the reference's own kernels (test infrastructure).

`cases(seed)` draws solar-wind-like primitive states (CGS) and stencils that
reach every branch of the kernels: smooth and discontinuous WENO stencils,
all-zero and subnormal components (the normalisation's special paths), NaN
and infinite entries, detector inputs on both sides of eta_d = 0.02,
negative densities and pressures for the clamps, Roe states that fall back
to Rusanov, and basis matrices like the cubed sphere's.  `evaluate(L, prefix,
c)` runs one library's exports (prefix "orc" for the oracle, "ref" for the
reference pin) on those inputs and returns a dict of output arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle.pyoracle import dptr

C_MP = 1.67262192e-24
GAMMA = 5.0 / 3.0
ENTROPY = 0.3
ETA_D = 0.02


def _state(rng, n):
    s = np.empty((n, 8))
    s[:, 0] = 700 * C_MP * rng.uniform(0.05, 4, n)
    s[:, 1:4] = rng.normal(0, 3e7, (n, 3))
    s[:, 4] = 1e-7 * rng.uniform(0.01, 3, n)
    s[:, 5:8] = rng.normal(0, 1e-4, (n, 3)) * rng.choice([0.0, 1.0], (n, 1))
    return s


def _stencils(rng, n, width=6):
    """n stencils of `width` cells x 8 components, a mix of kinds."""
    out = np.empty((n, width, 8))
    kinds = rng.integers(0, 7, n)
    for q in range(n):
        base = _state(rng, 1)[0]
        x = np.arange(width)[:, None]
        k = kinds[q]
        if k == 0:    # smooth: small gradients and curvature
            out[q] = base * (1 + 1e-2 * rng.normal(size=8) * x + 1e-3 * rng.normal(size=8) * x * x)
        elif k == 1:  # a jump between two states
            other = _state(rng, 1)[0]
            cut = rng.integers(1, width)
            out[q] = np.where(x < cut, base, other)
        elif k == 2:  # independent cells
            out[q] = _state(rng, width)
        elif k == 3:  # zero components (unmagnetised, or one exactly zero)
            out[q] = base * (1 + 1e-2 * rng.normal(size=(width, 8)))
            out[q][:, 5:8] = 0.0
            out[q][:, rng.integers(1, 4)] = 0.0
        elif k == 4:  # subnormal and tiny scales in some components
            out[q] = base * (1 + 1e-2 * rng.normal(size=(width, 8)))
            out[q][:, 5] = rng.normal(size=width) * 1e-310
            out[q][:, 6] = rng.normal(size=width) * 1e-300
            out[q][:, 7] = np.where(x[:, 0] == rng.integers(0, width), 4e-320, 0.0)
        elif k == 5:  # one non-finite entry
            out[q] = base * (1 + 1e-2 * rng.normal(size=(width, 8)))
            out[q][rng.integers(0, width), rng.integers(0, 8)] = [np.nan, np.inf, -np.inf][rng.integers(0, 3)]
        else:         # sign changes around zero (velocities, fields)
            out[q] = base * (1 + 1e-2 * rng.normal(size=(width, 8)))
            out[q][:, 1:4] = rng.normal(0, 1e5, (width, 3))
            out[q][:, 5:8] = rng.normal(0, 1e-6, (width, 3))
    return out, kinds


def _basis(rng, n):
    """Cubed-sphere-like bases: a rotation times a near-identity stretch."""
    out = np.empty((n, 3, 3))
    for q in range(n):
        Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        if np.linalg.det(Q) < 0:
            Q[:, 0] = -Q[:, 0]
        out[q] = Q @ (np.eye(3) + 0.2 * rng.normal(size=(3, 3)))
        if np.linalg.det(out[q]) < 0:
            out[q][:, 0] = -out[q][:, 0]
    return out


def cases(seed: int, n: int = 512) -> dict:
    rng = np.random.default_rng(seed)
    c = {}
    c["stencil"], c["stencil_kind"] = _stencils(rng, n)
    c["dx2"] = rng.choice([1.0 / 32 ** 2, 1.0 / 64 ** 2, 1.0 / 192 ** 2], n)
    # detector: a cell and its six neighbours, perturbations from 1e-5 to 30 %
    amp = 10 ** rng.uniform(-5, np.log10(0.3), n)
    base = _state(rng, n)
    c["jameson"] = base[:, None, :] * (1 + amp[:, None, None] * rng.normal(size=(n, 7, 8)))
    c["jameson"][rng.random(n) < 0.05, 3, 0] = np.nan
    # corrections: values, Laplacians, flags (including the 0.5 boundary)
    c["corr_val"] = _state(rng, n)
    c["corr_lap"] = c["corr_val"] * rng.normal(0, 0.1, (n, 8))
    c["corr_theta"] = rng.choice([0.0, 1.0, 0.5, 0.5000001, 0.4999999], n)
    # select: WENOZ and fallback states with non-positive density / pressure
    sel = _state(rng, 4 * n).reshape(n, 4, 8)
    bad = rng.random((n, 4)) < 0.3
    sel[:, :, 0] = np.where(bad, -np.abs(sel[:, :, 0]) * rng.choice([0.0, 1.0, 1e-4], (n, 4)), sel[:, :, 0])
    bad = rng.random((n, 4)) < 0.3
    sel[:, :, 4] = np.where(bad, -np.abs(sel[:, :, 4]) * rng.choice([0.0, 1.0, 1e-6], (n, 4)), sel[:, :, 4])
    sel[rng.random(n) < 0.05, 0, 4] = np.nan
    c["select"] = sel
    c["select_theta"] = rng.choice([0.0, 1.0], n)
    # mapped-flux lines
    m = 64
    c["line"] = rng.normal(size=(6, 3, m)) * rng.choice([1.0, 1e-3, 1e5], (6, 1, 1))
    # point primitives and physical flux
    u = _state(rng, n)
    u[:, 1:4] *= u[:, :1]
    u[:, 0] = np.where(rng.random(n) < 0.2, u[:, 0] * rng.choice([1e-3, 0.0, -1.0], n), u[:, 0])
    c["cons"] = u
    c["prim"] = _state(rng, n)
    c["energy"] = np.abs(rng.normal(size=(n, 3))) * 1e-7
    c["energy"][:, 2] *= rng.choice([-1.0, 1.0], n)
    c["centering"] = rng.integers(0, 3, n).astype(np.int32)
    # mapped / factored Roe on face states in the native basis
    wl, wr = _state(rng, n), _state(rng, n)
    close = rng.random(n) < 0.3
    wr[close] = wl[close] * (1 + rng.normal(0, 1e-3, (close.sum(), 8)))
    wr[rng.random(n) < 0.03, 0] = -1.0e-30
    c["roe_wl"], c["roe_wr"] = wl, wr
    c["roe_basis"] = _basis(rng, n)
    c["roe_area"] = rng.uniform(0.5, 3.0, n)
    c["roe_dir"] = rng.integers(0, 3, n).astype(np.int32)
    # usable-state check
    us = _state(rng, n)
    kind = rng.integers(0, 5, n)
    us[kind == 1, 0] = 1.67262192e-24 / 100.0 * (1 - 1e-12)
    us[kind == 2, 4] = -1e-30
    us[kind == 3, rng.integers(0, 8)] = np.nan
    us[kind == 4, 0] = 1.67262192e-24 / 100.0
    c["usable"] = us
    return c


def evaluate(L: C.CDLL, prefix: str, c: dict) -> dict:
    f = lambda name: getattr(L, f"{prefix}_{name}")  # noqa: E731
    n = c["stencil"].shape[0]
    out = {k: np.zeros((n, 8)) for k in ("wenoz_l", "wenoz_r", "weno3_l", "weno3_r", "plm_l", "plm_r")}
    out["norm6"] = np.zeros((n, 6 * 8))
    out["norm6_scale"] = np.zeros((n, 8))
    out["norm4"] = np.zeros((n, 4 * 8))
    out["norm4_scale"] = np.zeros((n, 8))
    for q in range(n):
        st = np.ascontiguousarray(c["stencil"][q])
        st4 = np.ascontiguousarray(st[1:5])
        for a, b, fn, args in (("wenoz_l", "wenoz_r", "berta_wenoz", (st,)),
                               ("weno3_l", "weno3_r", "berta_weno3", (st4, float(c["dx2"][q]))),
                               ("plm_l", "plm_r", "berta_plm", (st4,))):
            l, r = np.zeros(8), np.zeros(8)
            f(fn)(*[dptr(x) if isinstance(x, np.ndarray) else x for x in args], dptr(l), dptr(r))
            out[a][q], out[b][q] = l, r
        for comp in range(8):
            v6 = np.ascontiguousarray(st[:, comp])
            out["norm6_scale"][q, comp] = f("berta_normalize")(dptr(v6), 6)
            out["norm6"][q, comp * 6:(comp + 1) * 6] = v6
            v4 = np.ascontiguousarray(st4[:, comp])
            out["norm4_scale"][q, comp] = f("berta_normalize")(dptr(v4), 4)
            out["norm4"][q, comp * 4:(comp + 1) * 4] = v4
    out["jameson"] = np.array([f("berta_jameson")(dptr(np.ascontiguousarray(x)), ETA_D) for x in c["jameson"]])
    for key, fn in (("avg_to_point", "berta_avg_to_point"), ("flux_to_avg", "berta_flux_to_avg")):
        res = np.zeros((n, 8))
        for q in range(n):
            o = np.zeros(8)
            f(fn)(dptr(np.ascontiguousarray(c["corr_val"][q])), dptr(np.ascontiguousarray(c["corr_lap"][q])),
                  float(c["corr_theta"][q]), dptr(o))
            res[q] = o
        out[key] = res
    sl, sr = np.zeros((n, 8)), np.zeros((n, 8))
    for q in range(n):
        s4 = [np.ascontiguousarray(c["select"][q, k]) for k in range(4)]
        l, r = np.zeros(8), np.zeros(8)
        f("berta_select")(*[dptr(x) for x in s4], float(c["select_theta"][q]), dptr(l), dptr(r))
        sl[q], sr[q] = l, r
    out["select_l"], out["select_r"] = sl, sr
    line = c["line"]
    m = line.shape[2]
    for ncol in (1, 3):
        for both in (0, 1):
            arrs = [np.ascontiguousarray(line[k, :ncol]) for k in range(6)]
            o = np.zeros(m)
            f("berta_mapped_line")(ncol, both, *[dptr(a) for a in arrs], m, dptr(o))
            out[f"line_{ncol}_{both}"] = o
    res = np.zeros((n, 8))
    for q in range(n):
        o = np.zeros(8)
        f("sph_to_prim_raw")(dptr(np.ascontiguousarray(c["cons"][q])), dptr(o))
        res[q] = o
    out["sph_to_prim"] = res
    res = np.zeros((n, 8))
    for q in range(n):
        o = np.zeros(8)
        e = c["energy"][q]
        f("prim_flux")(dptr(np.ascontiguousarray(c["prim"][q])), float(e[0]), float(e[1]), float(e[2]), GAMMA,
                       int(c["centering"][q]), dptr(o))
        res[q] = o
    out["prim_flux"] = res
    floor = f("rho_floor")()
    for key, fn in (("mapped_roe", "mapped_roe"), ("factored_roe", "factored_roe")):
        res = np.zeros((n, 8))
        for q in range(n):
            o = np.zeros(8)
            A = np.ascontiguousarray(c["roe_basis"][q].reshape(-1))
            f(fn)(dptr(np.ascontiguousarray(c["roe_wl"][q])), dptr(np.ascontiguousarray(c["roe_wr"][q])), dptr(A),
                  float(c["roe_area"][q]), int(c["roe_dir"][q]), GAMMA, ENTROPY, floor, dptr(o))
            res[q] = o
        out[key] = res
    if prefix == "orc":
        out["usable"] = np.array([L.orc_usable_primitive(dptr(np.ascontiguousarray(w))) for w in c["usable"]],
                                 dtype=np.int32)
    else:
        out["usable"] = np.array([L.ref_usable_primitive(dptr(np.ascontiguousarray(w)), floor) for w in c["usable"]],
                                 dtype=np.int32)
    out["rho_floor"] = np.array([floor])
    return out
