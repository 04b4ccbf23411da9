"""The oracle's fourth-order level step on the CPU: the seam interpolation of
Cartesian averages converges at fourth order, constant states survive the
Cartesian conversion, and the flux register + reflux make the panel seams
conservative (src/MHD_AMR.H:1478-1497: each side takes the mean flux).

The seam weights and the deriv3case / AMatrix restatements are this
project's (Proto is unvendored), so these are property checks, not pins.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle as po

PERM = [[1, 2, 0], [1, 2, 0], [1, 0, 2], [0, 1, 2], [1, 0, 2], [0, 1, 2]]
SIGN = [[1, -1, -1], [1, 1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1], [-1, -1, 1]]
C_MP = 1.67262192e-24


def unit(b, x1, x2):
    a = np.tan(-np.pi / 4 + np.pi / 2 * x1)
    c = np.tan(-np.pi / 4 + np.pi / 2 * x2)
    rho = np.sqrt(1 + a * a + c * c)
    q = [1 / rho, a / rho, c / rho]
    return [SIGN[b][k] * q[PERM[b][k]] for k in range(3)]


def smooth(X):
    x, y, z = X
    return np.sin(1.3 * x + 0.7 * y - 0.4 * z) + 0.5 * x * y * z


def exact_averages(na, ga, f=smooth):
    """Cell averages of f over every cell of the extended panel grids
    [-ga, na+ga)^2 (6-point Gauss-Legendre per direction), [6][k][j]."""
    gx, gw = np.polynomial.legendre.leggauss(6)
    gx, gw = 0.5 * (gx + 1), 0.5 * gw
    h = 1.0 / na
    x = (np.arange(-ga, na + ga)[:, None] + gx[None, :]) * h
    out = np.zeros((6, na + 2 * ga, na + 2 * ga))
    for b in range(6):
        F = f(unit(b, x[:, None, :, None], x[None, :, None, :]))
        out[b] = np.einsum("jkpq,p,q->kj", F, gw, gw)
    return out


def seam_error(na, nr=2):
    O = po.OracleLevelO4(po.make_params(nr=nr, na=na, spatial_order=4, riemann_solver=2))
    ga = O.ga
    nA = na + 2 * ga
    ex = exact_averages(na, ga)
    valid = np.zeros((nA, nA), bool)
    valid[ga:ga + na, ga:ga + na] = True
    # an admissible state (positive density and thermal energy) whose z
    # momentum is the smooth test function
    cart = np.zeros((6, 8, nA, nA, nr))
    cart[:, 0][:, valid, :] = 2.0 + ex[:, valid, None]
    cart[:, 3][:, valid, :] = ex[:, valid, None]
    cart[:, 4][:, valid, :] = 100.0
    cart = np.ascontiguousarray(cart.reshape(-1))
    O.seams(cart)
    got = cart.reshape(6, 8, nA, nA, nr)[:, 3, :, :, nr - 1]
    return np.abs(got - ex)[:, ~valid].max()


def test_seam_interpolation_is_fourth_order():
    e16, e32 = seam_error(16), seam_error(32)
    assert e32 < 2e-5
    assert e16 / e32 > 12.0, (e16, e32)


def test_seam_ghosts_at_a_jump_stay_admissible():
    """A density jump of 1:100 next to the seams: the fourth-order stencil
    undershoots below zero there, and those ghosts take the average of the
    donor cell that contains their centre; every ghost stays admissible."""
    na, nr = 16, 2
    O = po.OracleLevelO4(po.make_params(nr=nr, na=na, spatial_order=4, riemann_solver=2))
    ga = O.ga
    nA = na + 2 * ga
    valid = np.zeros((nA, nA), bool)
    valid[ga:ga + na, ga:ga + na] = True
    rng = np.random.default_rng(4)
    rho = np.where(rng.random((6, nA, nA)) < 0.5, 1.0, 100.0)
    cart = np.zeros((6, 8, nA, nA, nr))
    cart[:, 0][:, valid, :] = rho[:, valid, None]
    cart[:, 1][:, valid, :] = 3.0 * rho[:, valid, None]
    cart[:, 4][:, valid, :] = 1000.0 * rho[:, valid, None]
    before = cart.copy()
    flat = np.ascontiguousarray(cart.reshape(-1))
    O.seams(flat)
    out = flat.reshape(6, 8, nA, nA, nr)
    ghosts = out[:, :, ~valid, :]
    rho_g = ghosts[:, 0]
    thermal = ghosts[:, 4] - 0.5 * ghosts[:, 1] ** 2 / rho_g
    assert np.isfinite(ghosts).all()
    assert (rho_g > 0).all() and (thermal >= 0).all()
    # some ghosts took a donor cell's average: exactly one of the two levels
    donor = np.isin(rho_g, [1.0, 100.0])
    assert donor.sum() > 0
    np.testing.assert_array_equal(out[:, :, valid, :], before[:, :, valid, :])


def test_constant_cartesian_state_is_preserved():
    nr, na = 6, 16
    O = po.OracleLevelO4(po.make_params(nr=nr, na=na, spatial_order=4, riemann_solver=2))
    geo = po.OracleLevel(po.make_params(nr=nr, na=na))
    det = geo.geometry(4).reshape(6, na, na)
    U = np.array([1.0, 0.3, -0.2, 0.5, 2.0, 0.1, 0.2, -0.3])
    # JU = dVolr * <det A> * U for a constant Cartesian state
    rad = np.array([_dvolr(po.make_params(nr=nr, na=na), i) for i in range(nr)])
    ju = np.zeros((6, 8, na, na, nr))
    ju[:] = U[None, :, None, None, None] * det[:, None, :, :, None] * rad[None, None, None, None, :]
    cart = O.cartesian(np.ascontiguousarray(ju.reshape(-1))).reshape(6, 8, na + 12, na + 12, nr)
    err = np.abs(cart - U[None, :, None, None, None]).max()
    assert err < 1e-12, err


def _dvolr(p, i):
    r0, r1, C, dxi0 = p.inner_radius, p.outer_radius, p.radial_stretch, 1.0 / p.nr
    Rt = (r1 - r0) / np.expm1(C)
    rl = r0 + Rt * np.expm1(C * i * dxi0)
    rh = r0 + Rt * np.expm1(C * (i + 1) * dxi0)
    return (rh ** 3 - rl ** 3) / 3.0 / dxi0


def wind_state(nr, na, seed):
    """Native averages on the ghosted panels: a Parker-like wind with
    seeded angular structure (smooth across panels: a function of the
    Cartesian direction)."""
    rng = np.random.default_rng(seed)
    g = 5
    n = na + 2 * g
    p = po.make_params(nr=nr, na=na)
    r0, r1, C = p.inner_radius, p.outer_radius, p.radial_stretch
    Rt = (r1 - r0) / np.expm1(C)
    i = np.arange(-g, nr + g)
    r = r0 + Rt * np.expm1(C * (i + 0.5) / nr)
    s = r0 / r
    a = rng.normal(size=3)
    x = (np.arange(-g, na + g) + 0.5) / na
    us = np.zeros((6, 8, n, n, nr + 2 * g))
    for b in range(6):
        X = unit(b, x[None, :], x[:, None])
        ang = np.sin(a[0] * X[0] + a[1] * X[1] + a[2] * X[2])[:, :, None]
        rho = 700 * C_MP * s[None, None, :] ** 2 * (1 + 0.05 * ang)
        vr = 4e7 * (1 + 0.02 * ang)
        us[b, 0] = rho
        us[b, 1] = rho * vr
        us[b, 2] = rho * 1e5 * ang
        us[b, 3] = -rho * 2e5 * ang
        us[b, 5] = 5e-3 * s[None, None, :] ** 2
        us[b, 6] = 1e-5 * ang * s[None, None, :]
        pr = 1e-7 * s[None, None, :] ** (10 / 3)
        us[b, 4] = pr * 1.5 + 0.5 * rho * vr ** 2 + us[b, 5] ** 2 / (8 * np.pi)
    return np.ascontiguousarray(us.reshape(-1))


def test_reflux_makes_panel_seams_conservative():
    """After the register reflux the angular divergence telescopes over the
    whole sphere: total mass change = radial boundary fluxes only."""
    nr, na = 16, 16
    params = po.make_params(nr=nr, na=na, spatial_order=4, riemann_solver=2)
    O = po.OracleLevelO4(params)
    us = wind_state(nr, na, 7)
    assert np.isfinite(us).all()
    reg = O.register()
    k = O.rhs(us, reg, 1.0)
    assert np.isfinite(k).all()
    ng = (nr + 10) * (na + 10) ** 2
    radial = 0.0
    seam_before = k.reshape(6, 8, -1)[:, 0].sum()
    for b in range(6):
        box = po.HcBox()
        box.lo[:] = (0, 0, 0)
        box.hi[:] = (nr - 1, na - 1, na - 1)
        box.ghost = 5
        box.block = b
        rhs = np.zeros(8 * nr * na * na)
        f0 = np.zeros(8 * (nr + 1) * na * na)
        f1 = np.zeros(8 * nr * (na + 1) * na)
        f2 = np.zeros(8 * nr * na * (na + 1))
        O.base.box_rhs_o4(box, np.ascontiguousarray(us[b * 8 * ng:(b + 1) * 8 * ng]), rhs, [f0, f1, f2])
        F0 = f0.reshape(8, na, na, nr + 1)[0]
        radial += -nr * (F0[:, :, nr] - F0[:, :, 0]).sum()
    O.reflux(reg, k)
    total = k.reshape(6, 8, -1)[:, 0].sum()
    scale = np.abs(k.reshape(6, 8, -1)[:, 0]).sum()
    assert abs(total - radial) < 1e-12 * scale, (total, radial, seam_before)
    # without the reflux the seams leak mass at truncation level
    assert abs(seam_before - radial) > 1e3 * abs(total - radial)
