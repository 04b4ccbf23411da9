"""AMR Runge-Kutta stage logic on the CPU: the numpy restatement of the
tableaus (src/MHD_AMRRungeKutta.H:9-12) integrates dU/dt = k exactly for a
constant k and reproduces the classical RK4 update for a linear ODE, AvgDown
keeps a box's mean, and hc_amr_plan_create rejects restrictions that would
read or write outside their boxes before it touches the GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from heliocubed_b200 import _native as N
from oracle import pyoracle as po


@pytest.mark.parametrize("order", [3, 4])
def test_tableau_reproduces_rk_on_linear_ode(order):
    lam, dt = -0.7, 0.3
    u = np.array([1.0])
    stage = np.zeros(1)
    rk = [np.zeros(1) for _ in range(4)]
    for s in range(order):
        po.amr_rk_stage(u, stage, rk, order, s, dt)
        rk[s][...] = lam * stage
    po.amr_rk_stage(u, stage, rk, order, order, dt)
    z = lam * dt
    exact_poly = 1 + z + z * z / 2 + z ** 3 / 6 + (z ** 4 / 24 if order == 4 else 0)
    assert u[0] == pytest.approx(exact_poly, rel=1e-14)


def test_restrict_keeps_the_mean():
    rng = np.random.default_rng(0)
    fine = rng.normal(size=(8, 8, 6, 4))          # [c][k][j][i], fine box at (2, 4, 6)
    coarse = np.zeros((8, 5, 5, 5))               # coarse box at (0, 1, 2)
    po.amr_restrict(fine, (2, 4, 6), coarse, (0, 1, 2), (1, 2, 3), (2, 4, 6), (2, 2, 2))
    block = coarse[:, 1:5, 1:4, 1:3]
    assert np.allclose(block.mean(axis=(1, 2, 3)), fine.mean(axis=(1, 2, 3)), rtol=1e-14)
    assert (coarse[:, 0] == 0).all()


def _restrict(**kw):
    r = N.HcRestrictBox()
    r.fine, r.coarse = 8, 16  # never dereferenced by the validation
    d = dict(fine_lo=(0, 0, 0), fine_n=(8, 8, 8), coarse_lo=(0, 0, 0), coarse_n=(4, 4, 4), lo=(0, 0, 0),
             hi=(3, 3, 3), ratio=(2, 2, 2))
    d.update(kw)
    for k, v in d.items():
        getattr(r, k)[:] = list(v)
    return r


@pytest.mark.parametrize("bad", [dict(hi=(4, 3, 3)), dict(fine_n=(7, 8, 8)), dict(ratio=(0, 2, 2)),
                                 dict(lo=(-1, 0, 0)), dict(fine_lo=(1, 0, 0))])
def test_plan_rejects_out_of_box_restrictions(bad):
    lib = N.lib()
    arr = (N.HcRestrictBox * 1)(_restrict(**bad))
    out = C.c_void_p()
    rc = lib.hc_amr_plan_create(C.c_void_p(1), None, 0, arr, 1, C.byref(out))
    assert rc == -1 and not out.value
    assert b"restriction" in lib.hc_last_error()


def test_plan_rejects_boxes_without_arrays():
    lib = N.lib()
    b = N.HcRkBox()
    b.ncells = 10
    b.state = 8
    arr = (N.HcRkBox * 1)(b)
    out = C.c_void_p()
    assert lib.hc_amr_plan_create(C.c_void_p(1), arr, 1, None, 0, C.byref(out)) == -1


def test_reflux_oracle_signs_and_zero_correction():
    """Equal fine and coarse fluxes leave the rhs unchanged; a fine excess
    delta on a face corrects the coarse cell below it (fine above) by
    -scale * delta and the cell above it (fine below) by +scale * delta."""
    rng = np.random.default_rng(1)
    coarse_flux = rng.normal(size=(8, 4, 4, 5))            # faces of dir 0 over lo (0,0,0)
    fine_flux = np.zeros((8, 8, 8, 9))                     # fine faces of dir 0, ratio 2
    for I in range(5):
        fine_flux[:, :, :, 2 * I] = np.repeat(np.repeat(coarse_flux[:, :, :, I], 2, axis=1), 2, axis=2)
    rhs = rng.normal(size=(8, 4, 4, 4))
    before = rhs.copy()
    po.amr_reflux(fine_flux, (0, 0, 0), coarse_flux, (0, 0, 0), rhs, (0, 0, 0), (2, 0, 0), (2, 3, 3), (2, 2, 2), 0,
                  1, 3.0)
    assert np.allclose(rhs, before, atol=1e-15)
    fine_flux[:, :, :, 4] += 0.5        # fine faces at coarse face I = 2
    po.amr_reflux(fine_flux, (0, 0, 0), coarse_flux, (0, 0, 0), rhs, (0, 0, 0), (2, 0, 0), (2, 3, 3), (2, 2, 2), 0,
                  1, 3.0)
    assert np.allclose(rhs[:, :, :, 1] - before[:, :, :, 1], -1.5)
    assert np.array_equal(rhs[:, :, :, 2], before[:, :, :, 2])
    rhs2 = before.copy()
    po.amr_reflux(fine_flux, (0, 0, 0), coarse_flux, (0, 0, 0), rhs2, (0, 0, 0), (2, 0, 0), (2, 3, 3), (2, 2, 2), 0,
                  0, 3.0)
    assert np.allclose(rhs2[:, :, :, 2] - before[:, :, :, 2], 1.5)


def _patch(**kw):
    r = N.HcRefluxBox()
    r.fine_flux, r.coarse_flux, r.rhs = 8, 16, 24
    d = dict(fine_lo=(0, 0, 0), fine_n=(9, 8, 8), coarse_lo=(0, 0, 0), coarse_n=(5, 4, 4), rhs_lo=(0, 0, 0),
             rhs_n=(4, 4, 4), lo=(2, 0, 0), hi=(2, 3, 3), ratio=(2, 2, 2))
    d.update(kw)
    for k, v in d.items():
        getattr(r, k)[:] = list(v)
    r.dir, r.fine_side, r.scale = kw.get("dir", 0), kw.get("fine_side", 1), 1.0
    return r


@pytest.mark.parametrize("bad", [dict(hi=(2, 4, 3)), dict(fine_n=(9, 7, 8)), dict(rhs_lo=(2, 0, 0)),
                                 dict(lo=(0, 0, 0), hi=(0, 3, 3)), dict(ratio=(2, 0, 2))])
def test_reflux_patches_outside_their_boxes_are_rejected(bad):
    lib = N.lib()
    plan = C.c_void_p()
    assert lib.hc_amr_plan_create(C.c_void_p(1), None, 0, None, 0, C.byref(plan)) == 0
    try:
        arr = (N.HcRefluxBox * 1)(_patch(**bad))
        assert lib.hc_amr_plan_set_reflux(plan, arr, 1) == -1
        assert b"reflux patch" in lib.hc_last_error()
    finally:
        lib.hc_amr_plan_destroy(plan)
